"""Mara.measure.* and Mara.diffuse on the GPU against the compiled reference.

* The eight measures beyond mean_max_divB / max_lorentz_factor (Mara/mara.cpp:1954-2230) on
  the reference's states (tests/golden/diffuse.npz) and, live, on the measured primitive
  array an advance leaves behind (the reference's PrimitiveArray: the last RK stage's
  primitives).  Extremes are exact (each per-zone value is the reference's operation
  sequence); means to 1e-12 of the mean magnitude of their terms (the device sums in another
  order).
* Mara.diffuse (LaxDiffusion, Mara/hydro.cpp:205-283) after the reference's failing step and
  after set_failmask(1) in 2D and 1D, with the failure mask and the previous-state guess the
  device's own advances left: the state to the whole-step bound, 1e-10.
* A scheme change between advances (mgpu_reconfigure) keeps MaxLambda, the mask and the
  measured array, as the reference's process-wide solver does.
"""
import ast

import numpy as np
import pytest

from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu

NAMES = ["mean_cons", "mean_prim", "mean_energies", "mean_velocity", "mean_max_temperature",
         "mean_max_magnetic_field", "mean_max_sonic_mach", "mean_min_alfvenic_mach"]
STEP_TOL = 1e-10
SUM_TOL = 1e-12


def _scheme(kw):
    kw = dict(kw)
    n = kw.pop("n")
    x0, x1 = kw.pop("x0", None), kw.pop("x1", None)
    return Scheme(**kw), n, x0, x1


def _interior(P, nd, ng=3):
    sl = tuple(slice(ng, -ng) if d < nd else slice(None) for d in range(3))
    return P[sl].reshape(-1, 8)


def _term_scales(P, nd):
    """Mean |term| of each sum of mean_cons (P->U per zone) and mean_prim."""
    from oracle import PortOracle, Scheme as OScheme
    port = PortOracle(OScheme(n=(4, 4, 4)))
    Z = _interior(P, nd)
    U = np.array([port.prim_to_cons(z)[0] for z in Z])
    return np.abs(U).mean(0), np.abs(Z).mean(0)


def _gpu_measures(s):
    return {"mean_cons": s.mean_cons(), "mean_prim": s.mean_prim(),
            "mean_energies": list(s.mean_energies().values()), "mean_velocity": s.mean_velocity(),
            "mean_max_temperature": list(s.mean_max_temperature()),
            "mean_max_magnetic_field": list(s.mean_max_magnetic_field()),
            "mean_max_sonic_mach": list(s.mean_max_sonic_mach()),
            "mean_min_alfvenic_mach": list(s.mean_min_alfvenic_mach())}


def _check_measures(got, want, P, nd):
    su, sp = _term_scales(P, nd)
    for name in NAMES:
        a, b = np.array(got[name]), np.array(want[name])
        assert a.shape == b.shape, name
        if name == "mean_cons":
            assert (np.abs(a - b) <= SUM_TOL * su + 1e-300).all(), (name, a - b)
        elif name == "mean_prim":
            assert (np.abs(a - b) <= SUM_TOL * sp + 1e-300).all(), (name, a - b)
        elif name in ("mean_energies", "mean_velocity"):
            assert (np.abs(a - b) <= SUM_TOL * np.abs(b)).all(), (name, a - b)
        else:   # mean and extreme
            assert abs(a[0] - b[0]) <= SUM_TOL * abs(b[0]), (name, a, b)
            assert a[1] == b[1], (name, a, b)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_measures_of_reference_states(golden, k):
    g = golden("diffuse.npz")
    scheme, n, x0, x1 = _scheme(ast.literal_eval(str(g[f"c{k}_scheme"])))
    s = Solver(scheme, n, x0, x1)
    Q = np.ascontiguousarray(g[f"c{k}_Q"])
    s.set_primitive(Q)
    _check_measures(_gpu_measures(s), {nm: g[f"c{k}_{nm}"] for nm in NAMES}, Q, len(n))


def test_measures_read_the_last_stage_primitives():
    """After an advance the measures read the last RK stage's primitives, on both sides."""
    from ctf_b200 import ics
    from oracle import RefOracle, Scheme as OScheme
    n = (10, 8, 6)
    kw = dict(riemann="hlld", advance="rk3", extrap="plm")
    P0 = ics.turbulence_box(n, seed=41, vrms=0.3)
    ref = RefOracle(OScheme(n=n, **kw))
    try:
        s = Solver(Scheme(**kw), n)
        A = P0.copy()
        s.upload(P0.copy())
        assert ref.advance(A, 0.0) == 0 and s.advance(0.0) == 0
        for _ in range(2):
            dt = ref.get_timestep(0.3)
            assert ref.advance(A, dt) == 0 and s.advance(dt) == 0
        want = {nm: ref.measure(nm) for nm in NAMES}
        got = _gpu_measures(s)
        PA = ref.primitive_array().reshape(A.shape)
        # the two last-stage arrays agree to the step bound, so the measures to about that
        su, sp = _term_scales(PA, 3)
        for name in NAMES:
            a, b = np.array(got[name]), np.array(want[name])
            scale = su if name == "mean_cons" else sp if name == "mean_prim" else np.abs(b)
            assert (np.abs(a - b) <= 1e-10 * scale + 1e-300).all(), (name, a, b)
    finally:
        ref.close()


@pytest.mark.parametrize("k", [0, 1, 2])
def test_diffuse_matches_reference(golden, k):
    g = golden("diffuse.npz")
    kwd = ast.literal_eval(str(g[f"c{k}_scheme"]))
    scheme, n, x0, x1 = _scheme(kwd)
    s = Solver(scheme, n, x0, x1)
    s.upload(np.ascontiguousarray(g[f"c{k}_P0"]).copy())
    assert s.advance(0.0) == 0
    dts = g[f"c{k}_dts"]
    for i, dt in enumerate(dts):
        e = s.advance(float(dt))
        assert (e > 0) == (i == len(dts) - 1 and int(g[f"c{k}_failmask"]) < 0), (i, e)
    if int(g[f"c{k}_failmask"]) >= 0:
        s.set_failmask(int(g[f"c{k}_failmask"]))
    Q = np.ascontiguousarray(g[f"c{k}_P"]).copy()
    errors = s.diffuse_host(Q, float(g[f"c{k}_r"]))
    assert errors == int(g[f"c{k}_mask_out"].sum())
    want = g[f"c{k}_Q"]
    a, b = Q.reshape(-1, 8), want.reshape(-1, 8)
    for q in range(8):
        sc = np.abs(b[:, q]).max()
        assert np.abs(a[:, q] - b[:, q]).max() <= STEP_TOL * (sc if sc > 0 else 1.0), q
    assert np.abs(Q - g[f"c{k}_P"]).max() > 0            # the diffusion did something


def test_diffuse_without_failures_is_a_round_trip():
    """With an empty mask the diffusion adds nothing: the state is c2p(P->U(P)) from the
    measured array's guess, the primitives to c2p round-off."""
    from ctf_b200 import ics
    n = (8, 8, 8)
    s = Solver(Scheme(), n)
    P0 = ics.turbulence_box(n, seed=5)
    s.upload(P0.copy())
    assert s.advance(0.0) == 0
    Q = s.download()
    R = Q.copy()
    assert s.diffuse_host(R, 0.2) == 0
    assert np.abs(R - Q).max() <= 1e-12 * np.abs(Q).max()


def test_scheme_change_in_place_keeps_state_and_max_lambda():
    """set_riemann / set_advance / config_solver between advances, as the reference's crash
    ladders do: the solver continues from its state and MaxLambda (get_timestep after the
    change gives the reference's dt), and matches the reference over the next steps."""
    from ctf_b200 import ics
    from oracle import RefOracle, Scheme as OScheme
    n = (8, 8, 8)
    P0 = ics.turbulence_box(n, seed=44, vrms=0.3)
    ref = RefOracle(OScheme(n=n, riemann="hll", advance="rk2"))
    try:
        s = Solver(Scheme(riemann="hll", advance="rk2"), n)
        A = P0.copy()
        s.upload(P0.copy())
        assert ref.advance(A, 0.0) == 0 and s.advance(0.0) == 0
        dt = ref.get_timestep(0.3)
        assert ref.advance(A, dt) == 0 and s.advance(dt) == 0
        ref.dostring("Mara.set_riemann('hlld'); Mara.set_advance('rk3'); Mara.config_solver({theta=1.5}, true)")
        s.reconfigure(Scheme(riemann="hlld", advance="rk3", theta=1.5))
        for _ in range(2):
            dt = ref.get_timestep(0.3)
            assert abs(s.get_timestep(0.3) - dt) <= 1e-12 * dt
            assert ref.advance(A, dt) == 0 and s.advance(dt) == 0
        B = s.download()
        assert np.abs(B - A).max() <= STEP_TOL * np.abs(A).max()
        s.reconfigure(Scheme(riemann="hlld", advance="rk4"))       # RK4 registers allocated here
        assert s.advance(dt) == 0
        with pytest.raises(Exception):
            s.reconfigure(Scheme(precision="fp32"))                # needs a new solver
    finally:
        ref.close()
