"""The lean device layout (Scheme(layout='lean'), include/mara_gpu.h MGPU_LAYOUT_LEAN).

Its sweeps add their flux differences straight into the Runge-Kutta register and keep only
the six transverse face fields for flux-CT, so it holds a 1024^3 FP32-bulk box in 157 GB.
In FP64 it is the reference's arithmetic in another summation order, so it is held to the
reference's own golden steps at the parity bound; in FP32 bulk it is held to the FP64 path
at the FP32 bounds of test_gpu_fp32.py.
"""
import ast

import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import MaraError, Scheme, Solver, new_ou_field
from tests.test_gpu_fp32 import DIVB_TOL, L1_TOL, LINF_TOL, rel_errors, weighted_corner_div
from tests.test_gpu_parity import STEP_TOL, rel_linf

pytestmark = pytest.mark.gpu

LEAN_CASES = ["plm_hlld_rk2_8", "weno5_hlld_rk3_8", "plm_hllc_rk3_odd"]


def lean_solver(kw, precision="fp64"):
    kw = dict(kw)
    n = kw.pop("n")
    x0, x1 = kw.pop("x0", None), kw.pop("x1", None)
    return Solver(Scheme(precision=precision, layout="lean", **kw), n, x0, x1)


@pytest.mark.parametrize("case", LEAN_CASES)
def test_lean_fp64_matches_reference_steps(golden, case):
    """Every golden step from the reference's state and dt; MaxLambda is taken over the faces
    the update reads, a subset of the reference's, so it can only be smaller."""
    g = golden(f"step_{case}.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = lean_solver(kw)
    s.upload(g["P0"].copy())
    assert s.advance(0.0) == 0
    assert s.max_lambda <= g["max_lambda"][0] * (1 + 1e-12)
    assert s.max_lambda >= 0.9 * g["max_lambda"][0]
    for k, dt in enumerate(g["dts"]):
        if k > 0:
            s.upload(np.ascontiguousarray(g["states"][k - 1]))
        assert s.advance(float(dt)) == g["errors"][k + 1] == 0
        assert rel_linf(s.download(), g["states"][k]) <= STEP_TOL, k


def test_lean_fp64_chain_matches_standard_layout():
    """Twenty RK3 WENO5 steps of a non-cubic turbulence box with the dt chain: the lean and
    standard FP64 layouts agree to the parity bound, field included."""
    n = (24, 20, 16)
    P0 = ics.turbulence_box(n, seed=7, vrms=0.2)
    kw = dict(extrap="weno5", riemann="hlld", advance="rk3")
    a, b = Solver(Scheme(layout="lean", **kw), n), Solver(Scheme(**kw), n)
    for s in (a, b):
        s.upload(P0.copy())
        assert s.advance(0.0) == 0
    for _ in range(20):
        dt = b.get_timestep(0.3)
        assert a.advance(dt) == 0 and b.advance(dt) == 0
    assert rel_linf(a.download(), b.download()) <= STEP_TOL
    assert abs(a.get_timestep(0.3) - b.get_timestep(0.3)) <= 1e-3 * b.get_timestep(0.3)


def test_lean_failure_restores_the_state(golden):
    """The reference's failing HLLC step: the lean layout reports the same count, commits
    nothing, and its primitives are the c2p of the unchanged conserved state."""
    g = golden("step_hllc_fail_12.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = lean_solver(kw)
    before = np.ascontiguousarray(g["states"][1])
    s.upload(before.copy())
    e = s.advance(float(g["dts"][2]))
    assert e == g["errors"][3] and e > 0
    assert s.stats()["committed"] == 0
    assert rel_linf(s.download(), before) <= 1e-12
    # and the solver goes on from there: a smaller step commits
    assert s.advance(0.25 * float(g["dts"][2])) == 0


@pytest.mark.parametrize("learned", [False, True])
def test_lean_fp32_tracks_fp64(learned):
    """FP32 bulk in the lean layout against the plain FP64 path: the FP32 L1 target,
    the FP32 L-infinity bound, and flux-CT's weighted divergence held to round-off."""
    from ctf_b200 import train_c2p
    n = (32, 32, 32)
    kw = dict(extrap="weno5", riemann="hlld", advance="rk3")
    P0 = ics.turbulence_box(n, seed=31, vrms=0.3)
    ref = Solver(Scheme(**kw), n)
    ref.upload(P0.copy())
    assert ref.advance(0.0) == 0
    dt = ref.get_timestep(0.3)
    a = Solver(Scheme(precision="fp32", layout="lean", learned_c2p=learned, **kw), n)
    if learned:
        a.set_c2p_network(train_c2p.load())
    a.upload(P0.copy())
    for _ in range(10):
        assert a.advance(dt) == 0 and ref.advance(dt) == 0
    l1, linf = rel_errors(a.download(), ref.download(), 3)
    assert l1.max() <= L1_TOL, l1
    assert linf.max() <= LINF_TOL, linf
    drift = weighted_corner_div(a.download(), n) - weighted_corner_div(P0, n)
    assert np.abs(drift).max() / max(n) <= DIVB_TOL
    mean, mx = a.mean_max_divB_state()
    assert abs(mx) <= DIVB_TOL and abs(mean) <= DIVB_TOL


def test_lean_driving_matches_standard_layout():
    """OU driving after committed advances: the lean kick rebuilds the committed conserved
    state from the kicked primitives; FP64 lean and standard stay at the parity bound (the
    lean layout samples the field in FP32, so the bound is the field's rounding)."""
    n = (16, 16, 16)
    P0 = ics.turbulence_box(n, seed=3, vrms=0.1)
    field = new_ou_field(3, 0.5, 1.0, 3, 99)
    kw = dict(extrap="plm", riemann="hlld", advance="rk2")
    a, b = Solver(Scheme(layout="lean", **kw), n), Solver(Scheme(**kw), n)
    for s in (a, b):
        s.set_driving(field)
        s.upload(P0.copy())
        assert s.advance(0.0) == 0
    for step in range(4):
        dt = b.get_timestep(0.3)
        for s in (a, b):
            s.driving_advance(dt)
            s.driving_resample()
            assert s.advance(dt) == 0
    assert rel_linf(a.download(), b.download()) <= 1e-6
    assert abs(a.driving_power() - b.driving_power()) <= 1e-6 * b.driving_power()


def test_lean_range_transfers():
    """Slab-by-slab upload equals a whole upload (guards refilled from the interior); range
    downloads are slices of the whole download."""
    n = (12, 10, 8)
    P0 = ics.turbulence_box(n, seed=5)
    a = Solver(Scheme(layout="lean", precision="fp32"), n)
    b = Solver(Scheme(layout="lean", precision="fp32"), n)
    a.upload(P0.copy())
    flat = P0.reshape(-1, 8)
    junk = P0.copy()
    junk[:3] = 7.0                      # guard zones of the upload are ignored
    jflat = junk.reshape(-1, 8)
    slab = 10 * 8 * 14
    for z0 in range(0, flat.shape[0], slab):
        b.upload_range(jflat[z0:z0 + slab], z0)
    whole = a.download()
    assert np.array_equal(whole, b.download())
    assert np.array_equal(b.download_range(1000, 333), whole.reshape(-1, 8)[1000:1333])
    # PA holds FP32 bulk components; the field is FP64 exactly
    assert np.array_equal(whole[..., 5:], P0[..., 5:])


def test_lean_set_primitive_uploads_the_committed_state():
    """The stage array holds the committed primitives, so set_primitive (what Mara.init_prim
    ends with) uploads them: the measures read them and the next advance starts from them."""
    n = (8, 8, 8)
    P0 = ics.turbulence_box(n, seed=2)
    a, b = Solver(Scheme(layout="lean"), n), Solver(Scheme(layout="lean"), n)
    a.set_primitive(P0.copy())
    b.upload(P0.copy())
    assert np.array_equal(a.download(), b.download())
    assert a.max_lorentz_factor() == b.max_lorentz_factor()
    assert a.advance(0.0) == 0 and b.advance(0.0) == 0
    assert np.array_equal(a.download(), b.download())


def test_lean_rejections():
    with pytest.raises(MaraError):
        Solver(Scheme(layout="lean"), (16, 16))                      # 3D only
    with pytest.raises(MaraError):
        Solver(Scheme(layout="lean", godunov="plm-muscl"), (8, 8, 8))
    with pytest.raises(MaraError):
        Solver(Scheme(layout="lean", advance="rk4"), (8, 8, 8))
