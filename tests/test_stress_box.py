"""The high-magnetisation stress box (Lorentz factors log-uniform in [1, 10], magnetisation
log-uniform in [0.1, 10], p = 0.01; ctf_b200.ics.stress_box) on the compiled reference: its
own algorithm cannot advance the box -- the first step fails c2p in thousands of zones -- and
with its emergency reset (config_solver{ereset = true}, Mara/hydro.cpp:165-199) it advances
without errors.  The C restatement reproduces both bit for bit.  Runs without a GPU."""
import os

import numpy as np
import pytest

from ctf_b200 import ics
from oracle import REF_SO, PortOracle, RefOracle, Scheme

pytestmark = pytest.mark.skipif(not os.path.exists(REF_SO), reason="the compiled reference (oracle/_ref) is not built")

N = (24, 24, 24)
KW = dict(n=N, riemann="hlld", advance="rk3", extrap="plm")


def test_reference_fails_the_stress_box_on_the_first_step():
    P0 = ics.stress_box(N, seed=0)
    ref, port = RefOracle(Scheme(**KW)), PortOracle(Scheme(**KW))
    try:
        A, B = P0.copy(), P0.copy()
        assert ref.advance(A, 0.0) == 0 and port.advance(B, 0.0) == 0
        dt = ref.get_timestep(0.3)
        A1 = A.copy()
        e_ref = ref.advance(A, dt)
        assert e_ref == port.advance(B, dt)
        # failed zones counted once per guarded copy; more than a quarter of the 24^3 interior
        assert e_ref > 0.25 * np.prod(N)
        assert np.array_equal(A, A1)          # a failed step leaves the state unchanged
    finally:
        ref.close()


def test_reference_emergency_reset_advances_the_stress_box():
    P0 = ics.stress_box(N, seed=0)
    kw = dict(KW, ereset=True, preset=0.01, dreset=1.0)
    ref, port = RefOracle(Scheme(**kw)), PortOracle(Scheme(**kw))
    try:
        A, B = P0.copy(), P0.copy()
        assert ref.advance(A, 0.0) == 0 and port.advance(B, 0.0) == 0
        dt = ref.get_timestep(0.3)
        for _ in range(2):
            assert ref.advance(A, dt) == 0 and port.advance(B, dt) == 0
            assert np.array_equal(A, B)
        assert not np.array_equal(A, P0)
    finally:
        ref.close()
