"""Generate the golden vectors in tests/golden/ from the compiled reference.

Runs only where the reference sources are available (``make -C oracle ref`` builds
``oracle/_ref/libmara_ref.so`` from them); the fixtures it writes are committed so that the
tests need neither the reference nor its build on any other machine.

    python tests/golden/make_golden.py [name ...]     # all fixtures, or the named step cases

Fixtures (all float64, AoS primitive layout with 3 guard zones where a grid is involved):
  step_*.npz      whole-step runs through Mara.advance / Mara.get_timestep
  c2p.npz         Rmhd::ConsToPrim (ladder) and the two solvers on random states
  flux.npz        FluxAndEigenvalues on random prims, dims 1..3
  riemann_*.npz   IntercellFlux of HLL / HLLC / HLLD on random face pairs
  recon.npz       PLM (theta=2) and WENO5-FV (JS96, B08, SZ10) on random stencils
  c2p_paths.npz, riemann_hlld_paths.npz
                  states chosen by the branch the reference takes on them (path_fixtures)
  diffuse.npz     Mara.diffuse after a failed step / set_failmask, and Mara.measure.*
  divb.npz        measure.mean_max_divB / max_lorentz_factor on the step fixtures' states
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ctf_b200 import ics  # noqa: E402
from oracle import RefOracle, Scheme  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

STEP_CASES = {
    # name: (scheme kwargs, IC builder, steps, cfl)
    "plm_hlld_rk2_8": (dict(n=(8, 8, 8)), lambda: ics.turbulence_box((8, 8, 8), seed=11), 6, 0.3),
    "weno5_hlld_rk3_8": (dict(n=(8, 8, 8), extrap="weno5", advance="rk3"),
                         lambda: ics.turbulence_box((8, 8, 8), seed=12), 4, 0.3),
    "plm_hllc_rk3_odd": (dict(n=(9, 7, 5), riemann="hllc", advance="rk3"),
                         lambda: ics.turbulence_box((9, 7, 5), seed=13), 4, 0.3),
    "pcm_hll_rk4_6": (dict(n=(6, 6, 6), extrap="pcm", riemann="hll", advance="rk4"),
                      lambda: ics.turbulence_box((6, 6, 6), seed=14), 3, 0.3),
    "kh2d_plm_hllc_rk3": (dict(n=(24, 16), x0=(0.0, 0.0), x1=(1.0, 1.0), riemann="hllc",
                               advance="rk3"), lambda: ics.kh_box((24, 16), seed=15), 5, 0.3),
    "kh2d_weno5_hlld_rk2": (dict(n=(16, 12), x0=(0.0, 0.0), x1=(1.0, 1.0), extrap="weno5",
                                 advance="rk2"), lambda: ics.kh_box((16, 12), seed=16), 4, 0.3),
    "hllc_fail_12": (dict(n=(12, 12, 12), riemann="hllc", advance="rk3"),
                    lambda: ics.turbulence_box((12, 12, 12), seed=1), 3, 0.3),
    # CTU-Hancock (set_godunov('plm-muscl')): the healthy step of ctf-core/drvtrb.lua:296-302
    # (single, HLLD, theta 2, CFL 0.24) and its fallbacks, in 3D, 2D and 1D
    "ctu_plm_hlld_single_8": (dict(n=(8, 8, 8), godunov="plm-muscl", advance="single"),
                              lambda: ics.turbulence_box((8, 8, 8), seed=17), 6, 0.24),
    "ctu_hll_rk2_odd": (dict(n=(9, 7, 6), godunov="plm-muscl", riemann="hll", advance="rk2",
                             theta=1.25), lambda: ics.turbulence_box((9, 7, 6), seed=18), 4, 0.3),
    "ctu_kh2d_hllc_rk3": (dict(n=(16, 12), x0=(0.0, 0.0), x1=(1.0, 1.0), godunov="plm-muscl",
                               riemann="hllc", advance="rk3", theta=1.5),
                          lambda: ics.kh_box((16, 12), seed=19), 4, 0.3),
    "ctu_1d_hlld_single": (dict(n=(24,), x0=(0.0,), x1=(1.0,), godunov="plm-muscl",
                                advance="single"), lambda: _line((24,), seed=20), 6, 0.3),
    "ctu_fail_8": (dict(n=(8, 7, 6), godunov="plm-muscl", riemann="hllc", advance="rk2"),
                   lambda: ics.turbulence_box((8, 7, 6), seed=1, vrms=0.4), 6, 0.4),
    # a zone with p < 0 under config_solver{ereset}: the stage c2p resets it and the operator
    # runs on P->U of the repaired primitives
    "ctu_ereset_8": (dict(n=(8, 8, 8), godunov="plm-muscl", ereset=True, preset=0.5, dreset=2.0),
                     lambda: _bad_zone((8, 8, 8), seed=3), 3, 0.3),
}


def _bad_zone(n, seed):
    P = ics.turbulence_box(n, seed=seed)
    P[5, 5, 5, 1] = -1.0
    return P


def _line(n, seed):
    """A 1D box: the x line through a 3D turbulence box, guards included."""
    P = ics.turbulence_box((n[0], 4, 4), seed=seed, vrms=0.5)
    return np.ascontiguousarray(P[:, 3, 3].reshape(n[0] + 6, 1, 1, 8))


def step_fixture(name, kw, ic, steps, cfl):
    scheme = Scheme(**kw)
    ref = RefOracle(scheme)
    P0 = ic()
    P = P0.copy()
    errs = [ref.advance(P, 0.0)]
    ml = [ref.max_lambda]
    dts, states = [], []
    for _ in range(steps):
        dt = ref.get_timestep(cfl)
        dts.append(dt)
        e = ref.advance(P, dt)
        errs.append(e)
        ml.append(ref.max_lambda)
        states.append(P.copy())
    divb = [ref.mean_max_divB(s) for s in [P0] + states]
    wmax = [ref.max_lorentz_factor(s) for s in [P0] + states]
    ref.close()
    np.savez_compressed(os.path.join(OUT, f"step_{name}.npz"), P0=P0, states=np.stack(states),
                        dts=np.array(dts), errors=np.array(errs), max_lambda=np.array(ml),
                        divb=np.array(divb), wmax=np.array(wmax), cfl=cfl,
                        scheme=np.array(repr(kw)))
    print(f"step_{name}: errors {errs}")


def random_prims(rng, n, wmax=10.0, sigma_max=10.0, pmin=1e-3):
    """Random physical prim states spanning low/high Lorentz factor and magnetisation."""
    rho = np.exp(rng.uniform(np.log(0.1), np.log(10.0), n))
    pre = np.exp(rng.uniform(np.log(pmin), np.log(10.0), n))
    W = np.exp(rng.uniform(0, np.log(wmax), n))
    vdir = rng.standard_normal((n, 3))
    vdir /= np.linalg.norm(vdir, axis=1, keepdims=True)
    v = vdir * np.sqrt(1 - 1 / W ** 2)[:, None]
    h = 1 + 4.0 * pre / rho
    sigma = np.exp(rng.uniform(np.log(1e-3), np.log(sigma_max), n))
    bdir = rng.standard_normal((n, 3))
    bdir /= np.linalg.norm(bdir, axis=1, keepdims=True)
    B = bdir * np.sqrt(sigma * rho * h)[:, None]
    return np.concatenate([rho[:, None], pre[:, None], v, B], axis=1)


def function_fixtures():
    rng = np.random.default_rng(2024)
    ref = RefOracle(Scheme(n=(4, 4, 4)))
    # c2p ----------------------------------------------------------------------------------
    P = random_prims(rng, 600)
    U = np.array([ref.prim_to_cons(p)[0] for p in P])
    ladder = [ref.cons_to_prim(u, guess=np.zeros(8)) for u in U]
    guess = P * (1 + 1e-3 * rng.standard_normal(P.shape))
    solvers = {}
    for solver in (0, 1):
        for g in (0, 1):
            res = [ref.c2p_solve(u, solver, g, pg) for u, pg in zip(U, guess)]
            solvers[f"P_{solver}{g}"] = np.array([r[0] for r in res])
            solvers[f"err_{solver}{g}"] = np.array([r[1] for r in res])
            solvers[f"it_{solver}{g}"] = np.array([r[2] for r in res])
    np.savez_compressed(os.path.join(OUT, "c2p.npz"), P=P, U=U, guess=guess,
                        P_ladder=np.array([r[0] for r in ladder]),
                        err_ladder=np.array([r[1] for r in ladder]), **solvers)
    # flux + eigenvalues --------------------------------------------------------------------
    P = random_prims(rng, 400)
    F = np.zeros((3, len(P), 8))
    lam = np.zeros((3, len(P), 2))
    for d in range(3):
        for i, p in enumerate(P):
            f, ap, am = ref.flux(p, d + 1)
            F[d, i] = f
            lam[d, i] = ap, am
    np.savez_compressed(os.path.join(OUT, "flux.npz"), P=P, F=F, lam=lam)
    ref.close()
    # Riemann solvers ------------------------------------------------------------------------
    for solver in ("hll", "hllc", "hlld"):
        ref = RefOracle(Scheme(n=(4, 4, 4), riemann=solver))
        Pl = random_prims(rng, 300, wmax=3.0, sigma_max=3.0)
        Pr = Pl * (1 + 0.2 * rng.standard_normal(Pl.shape))
        Pr[:, 0:2] = np.abs(Pr[:, 0:2])
        vr = Pr[:, 2:5]
        sp = np.linalg.norm(vr, axis=1)
        Pr[:, 2:5] = np.where((sp > 0.95)[:, None], vr * (0.95 / sp)[:, None], vr)
        Pr[:60, 5] = Pl[:60, 5] = 0.0                            # Bn = 0 faces
        Pr[60:90, 5:8] = Pl[60:90, 5:8] = Pl[60:90, 5:8] * 1e-9  # near-degenerate field
        F = np.zeros((3, len(Pl), 8))
        err = np.zeros((3, len(Pl)), dtype=int)
        mls = np.zeros((3, len(Pl)))
        for d in range(3):
            for i in range(len(Pl)):
                ref.lib.ref_reset_max_lambda()
                f, e = ref.riemann(Pl[i], Pr[i], d + 1)
                F[d, i] = f
                err[d, i] = e
                mls[d, i] = ref.max_lambda
        np.savez_compressed(os.path.join(OUT, f"riemann_{solver}.npz"), Pl=Pl, Pr=Pr, F=F,
                            err=err, max_lambda=mls)
        ref.close()
    # reconstruction ------------------------------------------------------------------------
    V = rng.standard_normal((500, 5))
    V[:100] = np.cumsum(np.abs(V[:100]), axis=1)      # monotone stencils
    V[100:150, 2] += 10.0                              # extrema
    out = {"V": V}
    for IS in ("js96", "b08", "sz10"):
        ref = RefOracle(Scheme(n=(4, 4, 4), extrap="weno5", IS=IS))
        out[f"weno_c2r_{IS}"] = np.array([ref.reconstruct(v, 4) for v in V])
        out[f"weno_c2l_{IS}"] = np.array([ref.reconstruct(v, 5) for v in V])
        ref.close()
    ref = RefOracle(Scheme(n=(4, 4, 4), theta=2.0))
    out["plm_c2r"] = np.array([ref.reconstruct(v, 1) for v in V])
    out["plm_c2l"] = np.array([ref.reconstruct(v, 0) for v in V])
    ref.close()
    np.savez_compressed(os.path.join(OUT, "recon.npz"), **out)


def path_fixtures():
    """States chosen by the path the reference's algorithm takes on them, so that every
    branch is pinned one by one (the random fixtures above resolve almost all on the first):

    c2p_paths.npz          conserved states whose gamma-law ladder (Mara/rmhd.cpp:103-176)
                           resolves on rung 2 (Anton from the previous primitives), 3 (Noble
                           from the estimate) or 4 (Noble from the previous primitives), or on
                           none; `rung` is that class
    riemann_hlld_paths.npz face pairs on which HLLD (Mara/riemann_hlld-rmhd.cpp:199-277)
                           succeeds on its 2nd or 3rd pressure guess, or falls back to HLLC
                           after all three fail or after its HLL-state c2p fails; `path` is
                           1-3 (attempt), 4 (all failed) or 0 (HLL c2p failed)

    The class comes from the C restatement (oracle/port, bit-exact with the reference on every
    other fixture); the golden outputs come from the compiled reference."""
    from oracle import PortOracle
    rng = np.random.default_rng(77)
    port = PortOracle(Scheme(n=(4, 4, 4)))
    want = {2: 60, 3: 60, 4: 40, 0: 30}
    picked = {k: [] for k in want}
    while any(len(picked[k]) < want[k] for k in want):
        P = random_prims(rng, 2000, wmax=float(rng.choice([10, 100, 1000])),
                         sigma_max=float(rng.choice([10, 1e3, 1e5])), pmin=1e-8)
        for p in P:
            U, _ = port.prim_to_cons(p)
            g = p * (1 + float(rng.choice([1e-9, 1e-6, 1e-3])) * rng.standard_normal(8))
            r = [port.c2p_solve(U, s_, gg, g)[1] for s_, gg in ((0, 0), (0, 1), (1, 0), (1, 1))]
            k = next((i + 1 for i, e in enumerate(r) if e == 0), 0)
            if k in want and len(picked[k]) < want[k]:
                picked[k].append((U, g, k))
    rows = [x for k in (2, 3, 4, 0) for x in picked[k]]
    U = np.array([x[0] for x in rows])
    G = np.array([x[1] for x in rows])
    rung = np.array([x[2] for x in rows])
    ref = RefOracle(Scheme(n=(4, 4, 4)))
    ladder = [ref.cons_to_prim(u, guess=g) for u, g in zip(U, G)]
    solvers = {}
    for solver in (0, 1):
        for gm in (0, 1):
            res = [ref.c2p_solve(u, solver, gm, g) for u, g in zip(U, G)]
            solvers[f"P_{solver}{gm}"] = np.array([x[0] for x in res])
            solvers[f"err_{solver}{gm}"] = np.array([x[1] for x in res])
            solvers[f"it_{solver}{gm}"] = np.array([x[2] for x in res])
    ref.close()
    np.savez_compressed(os.path.join(OUT, "c2p_paths.npz"), U=U, guess=G, rung=rung,
                        P_ladder=np.array([x[0] for x in ladder]),
                        err_ladder=np.array([x[1] for x in ladder]), **solvers)
    print("c2p_paths: rungs", {k: int((rung == k).sum()) for k in want})

    port = PortOracle(Scheme(n=(4, 4, 4), riemann="hlld"))
    want = {2: 50, 3: 50, 4: 50, 0: 40}
    picked = {k: [] for k in want}
    while any(len(picked[k]) < want[k] for k in want):
        Pl = random_prims(rng, 500, wmax=float(rng.choice([2, 5, 20])),
                          sigma_max=float(rng.choice([1, 10, 100])), pmin=1e-4)
        Pr = Pl * (1 + float(rng.choice([0.05, 0.3, 1.0])) * rng.standard_normal(Pl.shape))
        Pr[:, 0:2] = np.abs(Pr[:, 0:2])
        vr = Pr[:, 2:5]
        sp = np.linalg.norm(vr, axis=1)
        Pr[:, 2:5] = np.where((sp > 0.99)[:, None], vr * (0.99 / sp)[:, None], vr)
        for i in range(len(Pl)):
            d = int(rng.integers(1, 4))
            port.riemann(Pl[i], Pr[i], d)
            k = port.stats.hlld_path
            if k in want and len(picked[k]) < want[k]:
                picked[k].append((Pl[i], Pr[i], d, k))
    rows = [x for k in (2, 3, 4, 0) for x in picked[k]]
    Pl = np.array([x[0] for x in rows])
    Pr = np.array([x[1] for x in rows])
    dims = np.array([x[2] for x in rows])
    path = np.array([x[3] for x in rows])
    ref = RefOracle(Scheme(n=(4, 4, 4), riemann="hlld"))
    F = np.zeros((len(rows), 8))
    err = np.zeros(len(rows), dtype=int)
    mls = np.zeros(len(rows))
    for i in range(len(rows)):
        ref.lib.ref_reset_max_lambda()
        F[i], err[i] = ref.riemann(Pl[i], Pr[i], int(dims[i]))
        mls[i] = ref.max_lambda
    ref.close()
    np.savez_compressed(os.path.join(OUT, "riemann_hlld_paths.npz"), Pl=Pl, Pr=Pr, dim=dims, path=path,
                        F=F, err=err, max_lambda=mls)
    print("riemann_hlld_paths:", {k: int((path == k).sum()) for k in want})


def diffuse_fixtures():
    """diffuse.npz: Mara.diffuse (Mara/mara.cpp:343-366) and the eight other Mara.measure.*
    (Mara/mara.cpp:1954-2230), from the compiled reference.

    Cases (prefix c<k>_): 0 -- the 12^3 HLLC/RK3 turbulence box whose third step fails c2p
    in one zone (its four copies): diffuse(P, 0.2) of the state before that step, with the
    reference's own FailureMask and PrimitiveArray after the failed advance; 1 -- a 2D
    Kelvin-Helmholtz box after one step with set_failmask(1) (diffusion on every face,
    flux-CT in 2D), r = 0.3; 2 -- a 1D line after one step, set_failmask(1), r = 0.5.
    Stored per case: scheme, P0 (the initial state), dts (the advances from it, after the
    priming advance(P0, 0)), P (the diffuse's input), mask, PA (what the diffuse reads), Q (the
    result), mask_out, and the measures of Q."""
    out = {}
    names = ["mean_cons", "mean_prim", "mean_energies", "mean_velocity", "mean_max_temperature",
             "mean_max_magnetic_field", "mean_max_sonic_mach", "mean_min_alfvenic_mach"]
    cases = [
        (dict(n=(12, 12, 12), riemann="hllc", advance="rk3"), lambda: ics.turbulence_box((12, 12, 12), seed=1),
         None, 0.2),
        (dict(n=(24, 16), x0=(0.0, 0.0), x1=(1.0, 1.0), riemann="hlld", advance="rk2"),
         lambda: ics.kh_box((24, 16), seed=31), 1, 0.3),
        (dict(n=(40,), x0=(0.0,), x1=(1.0,), riemann="hlld", advance="rk3"), lambda: _line((40,), seed=32), 1, 0.5),
    ]
    for k, (kw, ic, failmask, r) in enumerate(cases):
        ref = RefOracle(Scheme(**kw))
        P = ic()
        P0 = P.copy()
        ref.advance(P, 0.0)
        dts = []
        while True:
            dt = ref.get_timestep(0.3)
            dts.append(dt)
            Pb = P.copy()
            e = ref.advance(P, dt)
            if failmask is not None or e:
                break
            assert len(dts) < 10, "the failing step was not reached"
        if failmask is not None:
            ref.set_failmask(failmask)
            Pb = P.copy()
        mask, PA = ref.failure_mask(), ref.primitive_array()
        Q = Pb.copy()
        ref.diffuse(Q, r)
        out[f"c{k}_scheme"] = np.array(repr(kw))
        out[f"c{k}_failmask"] = np.array(-1 if failmask is None else failmask)
        out[f"c{k}_r"] = np.array(r)
        out[f"c{k}_dts"] = np.array(dts)
        out[f"c{k}_P0"] = P0
        out[f"c{k}_P"] = Pb
        out[f"c{k}_mask"] = mask
        out[f"c{k}_PA"] = PA.reshape(Pb.shape)
        out[f"c{k}_Q"] = Q
        out[f"c{k}_mask_out"] = ref.failure_mask()
        for nm in names:
            out[f"c{k}_{nm}"] = np.array(ref.measure(nm, Q))
        print(f"diffuse case {k}: mask {int(mask.sum())}, changed zones "
              f"{int((np.abs(Q - Pb).reshape(-1, 8).max(1) > 0).sum())}")
        ref.close()
    np.savez_compressed(os.path.join(OUT, "diffuse.npz"), **out)


if __name__ == "__main__":
    only = sys.argv[1:]          # fixture names to (re)generate; none: all of them
    for name, (kw, ic, steps, cfl) in STEP_CASES.items():
        if not only or name in only:
            step_fixture(name, kw, ic, steps, cfl)
    if not only or "functions" in only:
        function_fixtures()
    if not only or "paths" in only:
        path_fixtures()
    if not only or "diffuse" in only:
        diffuse_fixtures()
    total = sum(os.path.getsize(os.path.join(OUT, f)) for f in os.listdir(OUT) if f.endswith(".npz"))
    print(f"wrote {total / 1e6:.2f} MB of fixtures")
