"""The FP32-bulk path against the plain FP64 path (it has no reference oracle of its own).

FP32 carries reconstruction, the Riemann fluxes and the RK combine of rho, tau, S; FP64
carries the c2p Newton polish, the magnetic field with its constrained-transport update,
and the dt reduction.  Both paths advance the same box with the same fixed dt; the stated
bounds are the per-field relative L1 and L-infinity differences after the steps, and the
corner divergence of the FP32 path's (FP64) magnetic field.
"""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu

L1_TOL = 1e-5          # relative L1 per field (the FP32 density target, applied to every field)
LINF_TOL = 5e-3        # relative L-infinity per field (FP32 rounding at discontinuities)
DIVB_TOL = 1e-12       # corner divergence of B (as Mara.measure.mean_max_divB reports it)


def weighted_corner_div(P, n):
    """Corner-centred divergence of B with the 1/dx weights, on the unit box.

    Flux-CT keeps sum_d (four-point average of the d-differences of B_d) / dx_d constant
    at every corner.  Mara.measure.mean_max_divB (Mara/mara.cpp:2264-2324) drops the 1/dx_d,
    so on a box whose cells are not cubes its value drifts even in FP64; this weighted form
    is the one CT conserves on every box shape.
    """
    div = 0.0
    for d in range(3):
        D = np.diff(P[..., 5 + d], axis=d)
        for e in range(3):                 # average the d-difference over the corner's 4 edges
            if e != d:
                D = 0.5 * (D.take(range(D.shape[e] - 1), axis=e) + D.take(range(1, D.shape[e]), axis=e))
        div = div + D * n[d]
    return div


def interior(P, nd, ng=3):
    return P[tuple(slice(ng, -ng) if d < nd else slice(None) for d in range(3))]


def rel_errors(a, b, nd):
    a, b = interior(a, nd).reshape(-1, 8), interior(b, nd).reshape(-1, 8)
    l1, linf = [], []
    for q in range(8):
        s1, sinf = np.abs(b[:, q]).mean(), np.abs(b[:, q]).max()
        d = np.abs(a[:, q] - b[:, q])
        l1.append(d.mean() / s1 if s1 > 0 else d.mean())
        linf.append(d.max() / sinf if sinf > 0 else d.max())
    return np.array(l1), np.array(linf)


def run(prec, kw, n, P0, dt, steps):
    s = Solver(Scheme(precision=prec, **kw), n, None, None)
    s.upload(P0.copy())
    for _ in range(steps):
        assert s.advance(dt) == 0
    return s


# HLLC's star state divides by the normal field (w2 = (U_hll[B2] w1 - F_hll[B2]) / U_hll[B1],
# Mara/riemann_hllc-rmhd.cpp:96-110); where a random field's normal component is weak that
# amplifies the FP32 rounding of the face states (not of the solver: FP64 star-state
# arithmetic from the same FP32 states gives the same errors).  On the 3D turbulence boxes
# this leaves 5e-4 in the transverse velocities after 6 steps (density 9e-6), so that case
# carries HLLC_L1_TOL; the 2D KH boxes of the ensemble workload (uniform normal field on x faces) stay at
# 1e-6 (test_fp32_bulk_kelvin_helmholtz_2d).  HLLD has no such division.
HLLC_L1_TOL = 1e-3


@pytest.mark.parametrize("kw,n,steps,vrms,l1_tol", [
    (dict(extrap="plm", riemann="hlld", advance="rk2"), (32, 32, 32), 20, 0.3, L1_TOL),
    (dict(extrap="weno5", riemann="hlld", advance="rk3"), (32, 32, 32), 10, 0.3, L1_TOL),
    # HLLC on these boxes fails c2p within a few steps in the reference itself (the
    # step_hllc_fail_12 fixture; at 0.15c the bit-exact restatement fails at step 7), so
    # these cases stop earlier
    (dict(extrap="plm", riemann="hllc", advance="rk3"), (24, 20, 16), 6, 0.1, HLLC_L1_TOL),
    (dict(extrap="plm", riemann="hllc", advance="rk3"), (24, 20, 16), 6, 0.15, HLLC_L1_TOL),
])
def test_fp32_bulk_tracks_fp64_turbulence(kw, n, steps, vrms, l1_tol):
    P0 = ics.turbulence_box(n, seed=31, vrms=vrms)
    ref = Solver(Scheme(**kw), n)
    ref.upload(P0.copy())
    assert ref.advance(0.0) == 0
    dt = ref.get_timestep(0.3)
    a = run("fp32", kw, n, P0, dt, steps)
    b = run("fp64", kw, n, P0, dt, steps)
    l1, linf = rel_errors(a.download(), b.download(), 3)
    assert l1[0] <= L1_TOL, l1            # density: the FP32 target, every case
    assert l1.max() <= l1_tol, l1
    if l1_tol == L1_TOL:                  # HLLC: a few weak-normal-field zones differ by O(0.1)
        assert linf.max() <= LINF_TOL, linf
    # CT holds the weighted corner divergence at its initial value to round-off (scaled by
    # the smallest cell width, so the bound reads in the units of the reference's measure)
    drift = weighted_corner_div(a.download(), n) - weighted_corner_div(P0, n)
    assert np.abs(drift).max() / max(n) <= DIVB_TOL
    if len(set(n)) == 1:                  # cubic cells: the reference's measure is conserved too
        mean, mx = a.mean_max_divB_state()
        assert abs(mx) <= DIVB_TOL and abs(mean) <= DIVB_TOL


def test_fp32_bulk_kelvin_helmholtz_2d():
    kw = dict(extrap="plm", riemann="hllc", advance="rk3")
    n = (64, 64)
    P0 = ics.kh_box(n, seed=32)
    ref = Solver(Scheme(**kw), n)
    ref.upload(P0.copy())
    assert ref.advance(0.0) == 0
    dt = ref.get_timestep(0.3)
    a = run("fp32", kw, n, P0, dt, 20)
    b = run("fp64", kw, n, P0, dt, 20)
    A, B = interior(a.download(), 2).reshape(-1, 8), interior(b.download(), 2).reshape(-1, 8)
    # rho and p relative to themselves; v and B components relative to the mean |v| and
    # |B| (vy and By start as small perturbations of a flow along x)
    vs = np.sqrt((B[:, 2:5] ** 2).sum(1)).mean()
    bs = np.sqrt((B[:, 5:8] ** 2).sum(1)).mean()
    scale = np.array([np.abs(B[:, 0]).mean(), np.abs(B[:, 1]).mean(), vs, vs, vs, bs, bs, bs])
    l1 = np.abs(A - B).mean(0) / scale
    assert l1.max() <= L1_TOL, l1
    assert abs(a.mean_max_divB_state()[1]) <= DIVB_TOL


def test_fp32_device_dt_loop_matches_host_loop():
    """advance_async with the device-side dt (cfl * min_dx / MaxLambda of the previous
    step) follows the same sequence as a host loop of get_timestep + advance."""
    kw = dict(extrap="plm", riemann="hlld", advance="rk2", precision="fp32")
    n = (16, 16, 16)
    P0 = ics.turbulence_box(n, seed=33)
    a = Solver(Scheme(**kw), n)
    b = Solver(Scheme(**kw), n)
    for s in (a, b):
        s.upload(P0.copy())
        assert s.advance(0.0) == 0
    for _ in range(5):
        assert b.advance(b.get_timestep(0.3)) == 0
    a.advance_async(5, cfl=0.3)
    a.synchronize()
    assert np.array_equal(a.download(), b.download())
