"""The stress box on the GPU (16^3, PLM + HLLD + RK3): the FP64 path fails the first step in
the same zones as the reference's algorithm (the restatement, bit-exact with the reference on
this box), and with the emergency reset it advances.  With resets the box is chaotic in the
last bits: a one-ulp change of the libm calls of the wave-speed quartic alone moves the
restatement's state by 1e-4 (relative L1) after one step and 1e-2 after three (measured with
the perturbed-libm build of the restatement), because a zone that just fails or just passes
the c2p is reset or not.  The GPU's CUDA libm is such a change, so the reset path is held to
1e-3 after one step -- ten times that measured sensitivity -- not to the 1e-10 of the
well-conditioned boxes."""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme, Solver
from oracle import PortOracle, Scheme as OScheme

pytestmark = pytest.mark.gpu

N = (16, 16, 16)
KW = dict(riemann="hlld", advance="rk3", extrap="plm")
RESET = dict(ereset=True, preset=0.01, dreset=1.0)
ONE_ULP_L1_AFTER_ONE_STEP = 1e-4


def _rel_l1(a, b):
    a, b = a[3:-3, 3:-3, 3:-3].reshape(-1, 8), b[3:-3, 3:-3, 3:-3].reshape(-1, 8)
    return max(np.abs(a[:, q] - b[:, q]).mean() / np.abs(b[:, q]).mean() for q in range(8))


def test_fp64_fails_the_stress_box_like_the_reference():
    P0 = ics.stress_box(N, seed=0)
    port = PortOracle(OScheme(n=N, **KW))
    s = Solver(Scheme(**KW), N)
    B = P0.copy()
    s.upload(P0.copy())
    assert s.advance(0.0) == 0 and port.advance(B, 0.0) == 0
    dt = port.get_timestep(0.3)
    S1 = s.download()
    e = s.advance(dt)
    assert e == port.advance(B, dt) and e > 0
    assert np.array_equal(s.download(), S1)       # a failed step leaves the state unchanged


def test_fp64_emergency_reset_advances_the_stress_box():
    P0 = ics.stress_box(N, seed=0)
    port = PortOracle(OScheme(n=N, **KW, **RESET))
    s = Solver(Scheme(**KW, **RESET), N)
    B = P0.copy()
    s.upload(P0.copy())
    assert s.advance(0.0) == 0 and port.advance(B, 0.0) == 0
    dt = port.get_timestep(0.3)
    assert s.advance(dt) == 0 and port.advance(B, dt) == 0
    assert s.stats()["c2p_failed"] > 0            # zones were reset
    assert _rel_l1(s.download(), B) <= 10 * ONE_ULP_L1_AFTER_ONE_STEP
    for _ in range(2):
        assert s.advance(dt) == 0
    assert np.isfinite(s.download()).all()


@pytest.mark.parametrize("learned", [False, True])
def test_fp32_bulk_emergency_reset_advances_the_stress_box(learned):
    from ctf_b200.train_c2p import load as load_net
    P0 = ics.stress_box(N, seed=0)
    s = Solver(Scheme(precision="fp32", layout="lean", learned_c2p=learned, **KW, **RESET), N)
    if learned:
        s.set_c2p_network(load_net())
    s.upload(P0.copy())
    assert s.advance(0.0) == 0
    dt = s.get_timestep(0.3)
    for _ in range(3):
        assert s.advance(dt) == 0
    assert np.isfinite(s.download()).all()
