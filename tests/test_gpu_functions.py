"""Function-level parity: the CUDA device functions of the FP64 advance against the reference's
golden per-state vectors (tests/golden/, made by the compiled reference), one function at a
time, through the C ABI's mgpu_probe_* entry points.

Bit for bit where the arithmetic is the reference's operation sequence (P->U, the c2p
solvers and their iteration counts, PLM/WENO5 reconstruction, the physical flux).  Where the
fast wave speeds enter (the quartic's pow/acos/cos/sin from CUDA's libm, which differ from
glibc by a few ulp) the eigenvalues of the flux fixture are held to LIBM_REL.  A Riemann flux amplifies its wave speeds' rounding by up to |F| / (lambda+ - lambda-): the
fluxes and the faces' MaxLambda (where a near-degenerate pair of roots of the quartic can
amplify the libm difference too) are held to RIEMANN_REL (the whole-step bound) face by face,
and most faces (at least BITLIKE_SHARE of them) to 1e-14.
The path fixtures hold states on which the reference takes its rarer branches -- the c2p
ladder's rungs 2-4 and HLLD's second and third pressure guesses and its HLLC fallback -- so
each branch is pinned on the device, error codes and iteration counts included.
"""
import ctypes

import numpy as np
import pytest

from ctf_b200 import _lib

pytestmark = pytest.mark.gpu

GAMMA = 4.0 / 3.0
PFLOOR = -1.0          # the reference's default: pressure floor off
# relative bound where CUDA's libm enters (the quartic of the fast wave speeds)
LIBM_REL = 1e-12
# Riemann fluxes: every face within the whole-step bound, most faces within 1e-14
RIEMANN_REL = 1e-10
BITLIKE_SHARE = 0.9


def _dev(a, dtype):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def probe_c2p(mode, U, G):
    import torch
    lib = _lib.load()
    n = len(U)
    dU, dG = _dev(U, torch.float64), _dev(G, torch.float64)
    dP = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
    de = torch.zeros(n, dtype=torch.int32, device="cuda")
    di = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert lib.mgpu_probe_c2p(mode, GAMMA, PFLOOR, _ptr(dU), _ptr(dG), n, _ptr(dP), _ptr(de), _ptr(di)) == 0
    return dP.cpu().numpy(), de.cpu().numpy(), di.cpu().numpy()


def probe_p2c(P):
    import torch
    lib = _lib.load()
    n = len(P)
    dP = _dev(P, torch.float64)
    dU = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
    de = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert lib.mgpu_probe_prim_to_cons(GAMMA, _ptr(dP), n, _ptr(dU), _ptr(de)) == 0
    return dU.cpu().numpy(), de.cpu().numpy()


def probe_flux(P, dim):
    import torch
    lib = _lib.load()
    n = len(P)
    dP = _dev(P, torch.float64)
    dF = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
    dl = torch.zeros((n, 2), dtype=torch.float64, device="cuda")
    assert lib.mgpu_probe_flux(GAMMA, dim, _ptr(dP), n, _ptr(dF), _ptr(dl)) == 0
    return dF.cpu().numpy(), dl.cpu().numpy()


def probe_riemann(solver, Pl, Pr, dims):
    import torch
    lib = _lib.load()
    n = len(Pl)
    dl, dr = _dev(Pl, torch.float64), _dev(Pr, torch.float64)
    dd = _dev(np.broadcast_to(dims, (n,)), torch.int32)
    dF = torch.zeros((n, 8), dtype=torch.float64, device="cuda")
    de = torch.zeros(n, dtype=torch.int32, device="cuda")
    dm = torch.zeros(n, dtype=torch.float64, device="cuda")
    dh = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert lib.mgpu_probe_riemann(solver, 1, _ptr(dd), GAMMA, PFLOOR, _ptr(dl), _ptr(dr), n, _ptr(dF), _ptr(de),
                                  _ptr(dm), _ptr(dh)) == 0
    return dF.cpu().numpy(), de.cpu().numpy(), dm.cpu().numpy(), dh.cpu().numpy()


def probe_recon(op, V, theta=2.0, is_mode=0, sz10A=50.0):
    import torch
    lib = _lib.load()
    n = len(V)
    dV = _dev(V, torch.float64)
    do = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert lib.mgpu_probe_reconstruct(op, theta, is_mode, sz10A, _ptr(dV), n, _ptr(do)) == 0
    return do.cpu().numpy()


def face_rel(A, B):
    """Per-row max |A - B| / max |B| (rows of 8 components)."""
    den = np.abs(B).max(axis=1)
    return np.abs(A - B).max(axis=1) / np.where(den > 0, den, 1.0)


# ---- P -> U and the c2p ------------------------------------------------------------------

def test_prim_to_cons_bitexact(golden):
    g = golden("c2p.npz")
    U, e = probe_p2c(g["P"])
    assert not e.any()
    assert np.array_equal(U, g["U"])


def _check_c2p(g, guess_for_ladder):
    P, e, _ = probe_c2p(0, g["U"], guess_for_ladder)
    assert np.array_equal(e != 0, g["err_ladder"] != 0)
    assert np.array_equal(P, g["P_ladder"])
    for solver in (0, 1):
        for start in (0, 1):
            P, e, it = probe_c2p(1 + 2 * solver + start, g["U"], g["guess"])
            assert np.array_equal(e, g[f"err_{solver}{start}"]), (solver, start)
            assert np.array_equal(it, g[f"it_{solver}{start}"]), (solver, start)
            ok = e == 0
            assert np.array_equal(P[ok], g[f"P_{solver}{start}"][ok]), (solver, start)


def test_c2p_ladder_and_solvers_bitexact(golden):
    """Random states: the ladder from a zero previous state (the first RK stage's) and each
    solver from each starting point, with the reference's error codes and iteration counts."""
    g = golden("c2p.npz")
    _check_c2p(g, np.zeros_like(g["U"]))


def test_c2p_rungs_2_to_4_bitexact(golden):
    """States the reference's ladder resolves only on rung 2, 3 or 4, or not at all."""
    g = golden("c2p_paths.npz")
    assert set(np.unique(g["rung"])) == {0, 2, 3, 4}
    _check_c2p(g, g["guess"])
    # the rung each state needs is the rung the device's ladder used: rung r means the
    # solvers of rungs 1..r-1 failed from their starting points and rung r's succeeded
    errs = [probe_c2p(m, g["U"], g["guess"])[1] != 0 for m in (1, 2, 3, 4)]
    rung = np.where(~errs[0], 1, np.where(~errs[1], 2, np.where(~errs[2], 3, np.where(~errs[3], 4, 0))))
    assert np.array_equal(rung, g["rung"])


# ---- flux and fast speeds --------------------------------------------------------------

def test_flux_bitexact_and_speeds_within_libm(golden):
    g = golden("flux.npz")
    worst = 0.0
    for d in range(3):
        F, lam = probe_flux(g["P"], d + 1)
        assert np.array_equal(F, g["F"][d])
        rel = np.abs(lam - g["lam"][d]) / np.maximum(np.abs(g["lam"][d]), 1e-300)
        worst = max(worst, float(rel.max()))
    assert worst <= LIBM_REL, worst


# ---- Riemann solvers -------------------------------------------------------------------

@pytest.mark.parametrize("solver,name", [(0, "hll"), (1, "hllc"), (2, "hlld")])
def test_riemann_random_faces(golden, solver, name):
    g = golden(f"riemann_{name}.npz")
    for d in range(3):
        F, e, ml, _ = probe_riemann(solver, g["Pl"], g["Pr"], d + 1)
        assert np.array_equal(e, g["err"][d])
        ok = e == 0
        rel = face_rel(F[ok], g["F"][d][ok])
        assert rel.max() <= RIEMANN_REL, rel.max()
        assert (rel <= 1e-14).mean() >= BITLIKE_SHARE, (rel <= 1e-14).mean()
        mrel = np.abs(ml - g["max_lambda"][d]) / np.abs(g["max_lambda"][d])
        assert mrel.max() <= RIEMANN_REL and (mrel <= 1e-14).mean() >= BITLIKE_SHARE, mrel.max()


def test_hlld_second_third_guess_and_hllc_fallback(golden):
    """Faces on which the reference's HLLD needs its 2nd or 3rd pressure guess, or falls back
    to HLLC (all guesses failed, or its HLL-state c2p failed)."""
    g = golden("riemann_hlld_paths.npz")
    assert set(np.unique(g["path"])) == {0, 2, 3, 4}
    F, e, ml, used_hllc = probe_riemann(2, g["Pl"], g["Pr"], g["dim"])
    assert np.array_equal(e, g["err"])
    assert np.array_equal(used_hllc != 0, np.isin(g["path"], (0, 4)))
    ok = e == 0
    rel = face_rel(F[ok], g["F"][ok])
    assert rel.max() <= RIEMANN_REL, rel.max()
    assert (rel <= 1e-14).mean() >= BITLIKE_SHARE, (rel <= 1e-14).mean()
    mrel = np.abs(ml - g["max_lambda"]) / np.abs(g["max_lambda"])
    assert mrel.max() <= RIEMANN_REL and (mrel <= 1e-14).mean() >= BITLIKE_SHARE, mrel.max()


# ---- reconstruction --------------------------------------------------------------------

def test_reconstruct_bitexact(golden):
    g = golden("recon.npz")
    V = g["V"]
    assert np.array_equal(probe_recon(1, V), g["plm_c2r"])
    assert np.array_equal(probe_recon(0, V), g["plm_c2l"])
    for is_mode, IS in enumerate(("js96", "b08", "sz10")):
        assert np.array_equal(probe_recon(4, V, is_mode=is_mode), g[f"weno_c2r_{IS}"]), IS
        assert np.array_equal(probe_recon(5, V, is_mode=is_mode), g[f"weno_c2l_{IS}"]), IS


def test_probe_arguments_are_checked():
    lib = _lib.load()
    assert lib.mgpu_probe_c2p(9, GAMMA, PFLOOR, None, None, 0, None, None, None) == 1
    assert lib.mgpu_probe_flux(GAMMA, 4, None, 0, None, None) == 1
    assert lib.mgpu_probe_reconstruct(2, 2.0, 0, 50.0, None, 0, None) == 1
    assert lib.mgpu_probe_riemann(3, 1, None, GAMMA, PFLOOR, None, None, 0, None, None, None, None) == 1
