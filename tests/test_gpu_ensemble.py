"""Ensembles of uneven boxes (ctf_b200.ensemble) against single-box solvers.

Box b of an ensemble runs the single-box path's device arithmetic on its own arrays, with its
own dt, MaxLambda, error count and commit, so every comparison here is bit-for-bit: each
ensemble box against an mgpu_solver of the same box advanced the same way (and so, through
the single-box parity tests, against the reference)."""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.ensemble import Ensemble, kh_sizes
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu


def run_singles(scheme, sizes, states, steps, cfl=0.3, x0=None, x1=None):
    """Each box alone: advance(0), then `steps` advances at its own CFL step."""
    out, errs = [], []
    for b, (n, P0) in enumerate(zip(sizes, states)):
        s = Solver(scheme, n, None if x0 is None else x0[b], None if x1 is None else x1[b])
        s.upload(P0.copy())
        e = [s.advance(0.0)]
        for _ in range(steps):
            e.append(s.advance(s.get_timestep(cfl)))
        out.append(s.download())
        errs.append(e)
        s.close()
    return out, errs


def run_ensemble(scheme, sizes, states, steps, cfl=0.3, graph=True, nsteps_per_call=1, x0=None, x1=None):
    E = Ensemble(scheme, sizes, x0, x1)
    for b, P0 in enumerate(states):
        E.upload(b, P0)
    E.advance(dt=0.0, graph=graph)
    errs = [list(E.errors())]
    done = 0
    while done < steps:
        k = min(nsteps_per_call, steps - done)
        E.advance(cfl=cfl, nsteps=k, graph=graph)
        done += k
        errs.append(list(E.errors()))
    out = [E.download(b) for b in range(E.nb)]
    return E, out, errs


def kh_states(sizes, seed=0):
    return [ics.kh_box(n, seed=seed + b) for b, n in enumerate(sizes)]


def kh_l1(a, b):
    """Per-field L1 difference of 2D KH states: rho and p relative to themselves, v and B
    components relative to the mean |v| and |B| (vy and By start as small perturbations)."""
    A, B = a[3:-3, 3:-3].reshape(-1, 8), b[3:-3, 3:-3].reshape(-1, 8)
    vs = np.sqrt((B[:, 2:5] ** 2).sum(1)).mean()
    bs = np.sqrt((B[:, 5:8] ** 2).sum(1)).mean()
    scale = np.array([np.abs(B[:, 0]).mean(), np.abs(B[:, 1]).mean(), vs, vs, vs, bs, bs, bs])
    return np.abs(A - B).mean(0) / scale


def test_uneven_kh_boxes_match_single_solvers_fp64():
    """FP64 (compiled with --fmad=false in both translation units) is bit-identical."""
    sizes = [(24, 20), (32, 32), (16, 40), (48, 24), (20, 20), (36, 28)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3")
    states = kh_states(sizes, seed=3)
    ref, ref_err = run_singles(scheme, sizes, states, 6)
    E, got, errs = run_ensemble(scheme, sizes, states, 6)
    assert all(e == 0 for e in sum(ref_err, []))
    assert all(e == 0 for e in sum(errs, []))
    for b in range(len(sizes)):
        assert np.array_equal(got[b], ref[b]), (b, np.abs(got[b] - ref[b]).max())


@pytest.mark.parametrize("steps,tol", [(1, 1e-6), (6, 1e-3)])
def test_uneven_kh_boxes_track_single_solvers_fp32(steps, tol):
    """FP32-bulk kernels of the ensemble and of the single-box path are compiled separately
    with FMA contraction on, so they may round differently: after one step they agree to
    1e-6; over six steps HLLC's division by the (small, growing) normal field on y faces
    amplifies those roundings to ~2e-4 in places (the HLLC bound of test_gpu_fp32.py)."""
    sizes = [(24, 20), (32, 32), (16, 40), (48, 24), (20, 20), (36, 28)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3", precision="fp32")
    states = kh_states(sizes, seed=3)
    ref, ref_err = run_singles(scheme, sizes, states, steps)
    E, got, errs = run_ensemble(scheme, sizes, states, steps)
    assert all(e == 0 for e in sum(ref_err, []))
    assert all(e == 0 for e in sum(errs, []))
    for b in range(len(sizes)):
        l1 = kh_l1(got[b], ref[b])
        assert l1.max() <= tol, (b, l1)


def test_3d_weno5_hlld_rk4_boxes_with_extents():
    sizes = [(12, 10, 8), (8, 8, 8), (10, 14, 9)]
    x0 = [(0.0, 0.0, 0.0), (-1.0, 0.0, 0.5), (0.0, 0.0, 0.0)]
    x1 = [(1.0, 1.0, 1.0), (1.0, 2.0, 1.0), (0.5, 1.0, 2.0)]
    scheme = Scheme(extrap="weno5", riemann="hlld", advance="rk4")
    states = [ics.turbulence_box(n, seed=60 + b, vrms=0.2) for b, n in enumerate(sizes)]
    ref, _ = run_singles(scheme, sizes, states, 3, x0=x0, x1=x1)
    _, got, errs = run_ensemble(scheme, sizes, states, 3, x0=x0, x1=x1)
    assert all(e == 0 for e in sum(errs, []))
    for b in range(len(sizes)):
        assert np.array_equal(got[b], ref[b]), b


def test_graph_replay_and_multistep_graph_match_direct_launches():
    sizes = [(20, 24), (28, 16), (40, 40)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3", precision="fp32")
    states = kh_states(sizes, seed=8)
    _, direct, _ = run_ensemble(scheme, sizes, states, 5, graph=False)
    _, graphed, _ = run_ensemble(scheme, sizes, states, 5, graph=True)
    _, multi, _ = run_ensemble(scheme, sizes, states, 5, graph=True, nsteps_per_call=5)
    for b in range(len(sizes)):
        assert np.array_equal(direct[b], graphed[b])
        assert np.array_equal(direct[b], multi[b])


def test_per_box_dt_array():
    sizes = [(24, 24), (16, 32)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk2")
    states = kh_states(sizes, seed=21)
    dts = [1.3e-3, 7.0e-4]
    E = Ensemble(scheme, sizes)
    for b, P in enumerate(states):
        E.upload(b, P)
    E.advance(dt=dts, nsteps=2)
    assert list(E.errors()) == [0, 0]
    for b, n in enumerate(sizes):
        s = Solver(scheme, n)
        s.upload(states[b].copy())
        assert s.advance(dts[b]) == 0 and s.advance(dts[b]) == 0
        assert np.array_equal(E.download(b), s.download())
        assert E.stats(b)["dt"] == dts[b]


def test_a_failing_box_leaves_the_others_committed(golden):
    """Box 0 is the reference's HLLC failure case (its third step fails c2p in 4 guarded
    zones, tests/golden/step_hllc_fail_12.npz); the other boxes succeed or fail on their own:
    each box's error counts, commit and state match its single-box run."""
    g = golden("step_hllc_fail_12.npz")
    sizes = [(12, 12, 12), (12, 12, 12), (10, 12, 14)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3")
    states = [g["P0"], ics.turbulence_box(sizes[1], seed=5, vrms=0.05, dBrms=0.02),
              ics.turbulence_box(sizes[2], seed=6, vrms=0.05, dBrms=0.02)]
    ref, ref_err = run_singles(scheme, sizes, states, 3)
    E, got, errs = run_ensemble(scheme, sizes, states, 3)
    assert [e[0] for e in errs] == list(g["errors"])
    assert [ref_err[b] for b in range(3)] == [[e[b] for e in errs] for b in range(3)]
    assert any(ref_err[b][-1] == 0 for b in range(3))   # at least one box commits its last step
    for b in range(3):
        assert E.stats(b)["committed"] == (1 if ref_err[b][-1] == 0 else 0)
        assert np.array_equal(got[b], ref[b]), b


def test_timing_and_autotune_leave_the_state_alone():
    sizes = kh_sizes(6, seed=2, lo=16, hi=64)
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3", precision="fp32")
    states = kh_states(sizes, seed=40)
    E = Ensemble(scheme, sizes)
    for b, P in enumerate(states):
        E.upload(b, P)
    E.advance(dt=0.0)
    E.advance(cfl=0.3)
    before = [E.download(b) for b in range(E.nb)]
    st_before = [E.stats(b) for b in range(E.nb)]
    dt = E.timesteps(0.3)
    ms = E.time_advance(dt, dict(zone_tile=512, face_tile=256, zone_ctas_per_sm=4, face_ctas_per_sm=2,
                                 c2p_ctas_per_sm=4), reps=2)
    assert ms > 0
    shape, best = E.autotune(dt, reps=1)
    assert best > 0 and E.launch == shape
    for b in range(E.nb):
        assert np.array_equal(E.download(b), before[b])
        assert E.stats(b) == st_before[b]
    # the tuned shape advances to the same state as the default one
    E.advance(cfl=0.3, nsteps=2)
    F = Ensemble(scheme, sizes)
    for b, P in enumerate(states):
        F.upload(b, P)
    F.advance(dt=0.0)
    F.advance(cfl=0.3, nsteps=3, graph=False)
    for b in range(E.nb):
        assert np.array_equal(E.download(b), F.download(b))


def test_tuning_cache(tmp_path):
    sizes = [(24, 24), (32, 16)]
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3", precision="fp32")
    E = Ensemble(scheme, sizes)
    for b, P in enumerate(kh_states(sizes, seed=50)):
        E.upload(b, P)
    path = str(tmp_path / "tune.json")
    first = E.tuned(1e-3, reps=1, cache=path)
    E.launch = dict(zone_tile=256, face_tile=128, zone_ctas_per_sm=2, face_ctas_per_sm=2, c2p_ctas_per_sm=2)
    again = E.tuned(1e-3, reps=1, cache=path)
    assert again == first and E.launch == first["launch"]
