"""Parity of the CUDA step (through the C ABI) with the reference.

Bar for the plain FP64 path: <= 1e-10 relative L-infinity against the reference's own CPU
advance (golden fixtures from the compiled reference, and the bit-exact C restatement for
sizes too large to commit), with dt and MaxLambda agreeing to round-off and identical error
counts.  In practice the FP64 kernels reproduce the reference's operation order and differ
only through CUDA's pow/acos/cos/sin in the wave-speed quartic, so the observed differences
are ~1e-15.
"""
import ast

import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme as GpuScheme, Solver
from oracle import PortOracle, Scheme as OracleScheme

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10        # relative L-infinity per primitive component (the FP64 parity target after 20 steps)
DT_TOL = 1e-12          # relative, dt and MaxLambda
# Fixtures whose reference result is itself ill-conditioned in libm: the 2D KH layer has
# nearly double roots in the fast-speed quartic, and tests/test_oracle_port.py measures
# that a one-ulp change of pow/acos/cos/sin moves the reference's own step result by
# 1.7e-7 (PLM+HLLC) and 5.5e-8 (WENO5+HLLD) there.  CUDA's transcendentals differ from
# glibc's by such ulps, so the bound for those fixtures is set from the measured
# sensitivity (x6) instead of 1e-10.
CASE_TOL = {"kh2d_plm_hllc_rk3": 1e-6, "kh2d_weno5_hlld_rk2": 1e-6, "ctu_kh2d_hllc_rk3": 3e-6}

STEP_CASES = ["plm_hlld_rk2_8", "weno5_hlld_rk3_8", "plm_hllc_rk3_odd", "pcm_hll_rk4_6",
              "kh2d_plm_hllc_rk3", "kh2d_weno5_hlld_rk2", "hllc_fail_12",
              # CTU-Hancock (set_godunov('plm-muscl'))
              "ctu_plm_hlld_single_8", "ctu_hll_rk2_odd", "ctu_kh2d_hllc_rk3", "ctu_1d_hlld_single",
              "ctu_fail_8", "ctu_ereset_8"]


def rel_linf(a, b):
    """max over components of max|a-b| / max|b| (absolute where the component is zero)."""
    a = a.reshape(-1, 8)
    b = b.reshape(-1, 8)
    out = 0.0
    for q in range(8):
        scale = np.abs(b[:, q]).max()
        d = np.abs(a[:, q] - b[:, q]).max()
        out = max(out, d / scale if scale > 0 else d)
    return out


def gpu_solver(kw, precision="fp64"):
    kw = dict(kw)
    n = kw.pop("n")
    x0 = kw.pop("x0", None)
    x1 = kw.pop("x1", None)
    return Solver(GpuScheme(precision=precision, **kw), n, x0, x1)


@pytest.mark.parametrize("case", STEP_CASES)
def test_golden_steps_with_reference_dt(golden, case):
    """Each step from the reference's own state and dt: the state after one GPU step
    matches the reference's within STEP_TOL; error counts match exactly."""
    g = golden(f"step_{case}.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = gpu_solver(kw)
    P = g["P0"].copy()
    s.upload(P)
    assert s.advance(0.0) == g["errors"][0]
    for k, dt in enumerate(g["dts"]):
        if k > 0:
            s.upload(np.ascontiguousarray(g["states"][k - 1]))
        e = s.advance(float(dt))
        assert e == g["errors"][k + 1], (k, e)
        if e == 0:
            out = s.download()
            err = rel_linf(out, g["states"][k])
            assert err <= CASE_TOL.get(case, STEP_TOL), (k, err)


@pytest.mark.parametrize("case", STEP_CASES)
def test_golden_chain(golden, case):
    """The whole chain as a driver runs it: prime with advance(P, 0), then dt from
    get_timestep (the one-step lag of MaxLambda) and advance, for every fixture step."""
    g = golden(f"step_{case}.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = gpu_solver(kw)
    s.upload(g["P0"].copy())
    assert s.advance(0.0) == g["errors"][0]
    dt_tol = CASE_TOL.get(case, DT_TOL)
    assert abs(s.max_lambda - g["max_lambda"][0]) <= dt_tol * g["max_lambda"][0]
    for k, dt_ref in enumerate(g["dts"]):
        dt = s.get_timestep(float(g["cfl"]))
        assert abs(dt - dt_ref) <= dt_tol * dt_ref, (k, dt, dt_ref)
        e = s.advance(dt)
        assert e == g["errors"][k + 1]
        if e:
            break
        assert abs(s.max_lambda - g["max_lambda"][k + 1]) <= dt_tol * g["max_lambda"][k + 1]
        assert rel_linf(s.download(), g["states"][k]) <= CASE_TOL.get(case, STEP_TOL)


@pytest.mark.parametrize("case", ["plm_hlld_rk2_8", "plm_hllc_rk3_odd", "kh2d_plm_hllc_rk3"])
def test_measures(golden, case):
    g = golden(f"step_{case}.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = gpu_solver(kw)
    for i, P in enumerate([g["P0"]] + list(g["states"])):
        s.set_primitive(np.ascontiguousarray(P))
        mean, mx = s.mean_max_divB()
        assert mx == g["divb"][i][1]
        assert abs(mean - g["divb"][i][0]) <= 1e-12 * max(abs(g["divb"][i][1]), 1e-300) + 1e-30
        assert s.max_lorentz_factor() == g["wmax"][i]


def test_turbulence_64_twenty_steps_vs_oracle():
    """The plain-FP64 parity target: the 64^3 turbulence box (rho = p = 1, Gamma 4/3,
    seeded v rms 0.3c, Bz = 1 + solenoidal perturbation rms 0.1), PLM theta 2 + HLLD + RK2,
    CFL 0.3, 20 steps with the reference's dt lag, against the bit-exact C restatement
    (pinned to the reference by tests/test_oracle_port.py)."""
    n = (64, 64, 64)
    P0 = ics.turbulence_box(n, seed=0)
    port = PortOracle(OracleScheme(n=n))
    s = Solver(GpuScheme(), n)
    Pc = P0.copy()
    s.upload(P0.copy())
    assert port.advance(Pc, 0.0) == 0
    assert s.advance(0.0) == 0
    worst = 0.0
    for k in range(20):
        dt_c = port.get_timestep(0.3)
        dt_g = s.get_timestep(0.3)
        assert abs(dt_g - dt_c) <= DT_TOL * dt_c, (k, dt_g, dt_c)
        assert port.advance(Pc, dt_c) == 0
        assert s.advance(dt_g) == 0
        worst = max(worst, rel_linf(s.download(), Pc))
    assert worst <= STEP_TOL, worst
    # corner divergence of B stays at round-off (the initial B is discretely solenoidal)
    s.set_primitive(s.download())
    assert abs(s.mean_max_divB()[1]) <= 1e-12


def test_advance_host_matches_device_path():
    """Mara.advance(buf, dt) semantics through mgpu_advance_host: copy in, step, copy out."""
    n = (10, 8, 6)
    P0 = ics.turbulence_box(n, seed=5)
    a = Solver(GpuScheme(), n)
    b = Solver(GpuScheme(), n)
    P = P0.copy()
    kz, e = a.advance_host(P, 0.0)
    assert e == 0 and kz > 0
    b.upload(P0.copy())
    b.advance(0.0)
    assert np.array_equal(P, b.download())


def test_failure_leaves_state_unchanged(golden):
    """A step whose c2p fails reports the reference's count and commits nothing."""
    g = golden("step_hllc_fail_12.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    s = gpu_solver(kw)
    before = np.ascontiguousarray(g["states"][1])
    s.upload(before.copy())
    e = s.advance(float(g["dts"][2]))
    assert e == g["errors"][3] and e > 0
    assert np.array_equal(s.download(), before)
    st = s.stats()
    assert st["committed"] == 0 and st["errors"] == e


def test_emergency_reset_matches_oracle():
    """config_solver{ereset=true}: failed zones get (dreset, preset, v=0, B) and the step
    commits; compared with the C restatement."""
    n = (12, 12, 12)
    kw = dict(riemann="hllc", advance="rk3", ereset=True, preset=0.5, dreset=2.0)
    P0 = ics.turbulence_box(n, seed=1)
    port = PortOracle(OracleScheme(n=n, **kw))
    s = Solver(GpuScheme(**kw), n)
    Pc = P0.copy()
    s.upload(P0.copy())
    port.advance(Pc, 0.0)
    s.advance(0.0)
    for _ in range(4):
        dt = port.get_timestep(0.3)
        assert port.advance(Pc, dt) == 0
        assert s.advance(dt) == 0
    assert rel_linf(s.download(), Pc) <= STEP_TOL


def test_bad_input_counts_like_oracle():
    """Host-side fault injection: a zone with p < 0 and one with NaN make the c2p fail;
    the error count (guard images included) equals the restatement's."""
    n = (8, 8, 8)
    P0 = ics.turbulence_box(n, seed=3)
    P0[5, 5, 5, 1] = -1.0
    P0[3, 4, 5, 0] = np.nan      # a zone next to the guard layer: counted with its images
    port = PortOracle(OracleScheme(n=n))
    s = Solver(GpuScheme(), n)
    Pc = P0.copy()
    s.upload(P0.copy())
    e_c = port.advance(Pc, 1e-3)
    e_g = s.advance(1e-3)
    assert e_g == e_c and e_g > 0
