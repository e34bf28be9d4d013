"""The Lua drop-in (ctf_b200/lua/lmara_gpu.c): the reference's `Mara` module surface on the
GPU step, driven by the same Lua driver script in the reference's own interpreter
(oracle/_ref) and in this project's host (ctf_b200/_lib/libmaralua.so)."""
import os

import numpy as np
import pytest

from ctf_b200 import ics

pytest.importorskip("ctf_b200.luahost")
from ctf_b200.luahost import LIB_PATH, LuaError, LuaHost  # noqa: E402

needs_host = pytest.mark.skipif(not os.path.exists(LIB_PATH), reason="libmaralua.so not built")

DRIVER = r"""
Mara.start()
Mara.set_fluid('rmhd')
Mara.set_eos('gamma-law', 4.0 / 3.0)
Mara.set_godunov('plm-split')
Mara.set_boundary('periodic')
Mara.set_riemann('{riemann}')
Mara.set_advance('{advance}')
Mara.config_solver({{extrap='{extrap}', theta=2.0}}, true)
Mara.set_domain({{0,0,0}}, {{1,1,1}}, {{{n0},{n1},{n2}}}, 8, 3)
local f = io.open('{inp}', 'rb'); local P = buffer.new_buffer(f:read('*a')); f:close()
local log = io.open('{out}.txt', 'w')
local kz, e = Mara.advance(P, 0.0)
log:write(string.format('%d\n', e))
for n = 1, {steps} do
  local dt = Mara.get_timestep(0.3)
  kz, e = Mara.advance(P, dt)
  log:write(string.format('%d %.17g\n', e, dt))
end
local dm, dx = Mara.measure.mean_max_divB()
log:write(string.format('%.17g %.17g %.17g\n', dm, dx, Mara.measure.max_lorentz_factor()))
log:close()
local g = io.open('{out}', 'wb'); g:write(tostring(P)); g:close()
Mara.close()
"""


def test_driver_script_runs_in_the_reference(tmp_path):
    """The driver script itself, in the reference's interpreter (CPU)."""
    n = (8, 6, 6)
    P0 = ics.turbulence_box(n, seed=72, vrms=0.2)
    P, lines = _run_driver(tmp_path, "ref", dict(riemann="hlld", advance="rk2", extrap="plm"), n, 2, P0)
    assert lines[0] == "0" and all(ln.split()[0] == "0" for ln in lines[1:3])
    assert np.isfinite(P).all() and np.abs(P - P0).max() > 0


@needs_host
def test_module_surface_without_a_gpu():
    """Table layout, names and the error behaviour of misuse (no device call is made)."""
    with LuaHost() as h:
        h.run(r"""
        assert(type(Mara.advance) == 'function' and type(Mara.get_timestep) == 'function')
        assert(type(Mara.measure.mean_max_divB) == 'function')
        local names = Mara.fluid.GetPrimNames()
        assert(#names == 8 and names[1] == 'rho' and names[8] == 'Bz')
        local ok, msg = pcall(Mara.set_fluid, 'euler')
        assert(not ok and msg:find('not provided by the GPU module'))
        ok, msg = pcall(Mara.set_fluid, 'plasma')
        assert(not ok and msg:find("no such fluid 'plasma'"))
        ok, msg = pcall(Mara.set_cooling)
        assert(not ok and msg:find('set_cooling is not provided'))
        ok, msg = pcall(Mara.diffuse)
        assert(not ok and msg:find('expected a buffer as argument 1'))
        ok, msg = pcall(Mara.measure.mean_cons)
        assert(not ok and msg:find('call Mara.start'))
        assert(type(Mara.measure.mean_min_alfvenic_mach) == 'function')
        assert(Mara.cooling_rate(0.5) == 0.0)
        Mara.start()
        Mara.set_riemann('hllc'); Mara.set_advance('rk3')
        Mara.config_solver({extrap='weno5', IS='b08', precision='fp32'}, true)
        ok, msg = pcall(Mara.set_riemann, 'roe')
        assert(not ok and msg:find("no such riemann solver 'roe'"))
        ok, msg = pcall(Mara.config_solver, {extrap='ppm'}, true)
        assert(not ok and msg:find("no such extrap 'ppm'"))
        ok, msg = pcall(Mara.advance, buffer.new_buffer(64), 0.0)
        assert(not ok and msg:find('need a domain to run this'))
        ok, msg = pcall(Mara.advance_device, 0.0)
        assert(not ok and msg:find('need a domain to run this'))
        assert(type(Mara.upload_primitive) == 'function' and type(Mara.download_primitive) == 'function')
        """)
        with pytest.raises(LuaError, match="boom"):
            h.run("error('boom')")


def _run_driver(tmp_path, which, kw, n, steps, P0):
    inp = tmp_path / "P0.bin"
    P0.astype(np.float64).tofile(inp)
    out = tmp_path / f"P_{which}.bin"
    code = DRIVER.format(inp=inp, out=out, steps=steps, n0=n[0], n1=n[1], n2=n[2], **kw)
    if which == "gpu":
        with LuaHost() as h:
            h.run(code)
    else:
        from oracle import RefOracle, Scheme
        ref = RefOracle(Scheme(n=n))
        ref.dostring(code)
        ref.close()
    lines = open(str(out) + ".txt").read().split("\n")
    return np.fromfile(out).reshape(P0.shape), lines


@needs_host
@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(riemann="hlld", advance="rk2", extrap="plm"),
                                dict(riemann="hllc", advance="rk3", extrap="weno5")])
def test_driver_script_matches_the_reference(tmp_path, kw):
    n = (12, 10, 8)
    P0 = ics.turbulence_box(n, seed=71, vrms=0.2)
    Pg, lg = _run_driver(tmp_path, "gpu", kw, n, 4, P0)
    Pr, lr = _run_driver(tmp_path, "ref", kw, n, 4, P0)
    # error counts exactly, dt to 1e-12, state to 1e-10
    for a, b in zip(lg[:5], lr[:5]):
        ea, eb = a.split(), b.split()
        assert ea[0] == eb[0]
        if len(ea) > 1:
            assert abs(float(ea[1]) - float(eb[1])) <= 1e-12 * float(eb[1])
    assert np.abs(Pg - Pr).max() <= 1e-10 * np.abs(Pr).max()
    # measures of the last stage's primitives: corner divergence (mean, max), max Lorentz factor
    mg, mr = [float(x) for x in lg[5].split()], [float(x) for x in lr[5].split()]
    assert abs(mg[0] - mr[0]) <= 1e-9 * abs(mr[1])
    assert abs(mg[1] - mr[1]) <= 1e-9 * abs(mr[1])
    assert abs(mg[2] - mr[2]) <= 1e-12 * mr[2]


# The same driver loop on a device-resident state: one upload, advance_device per step (no
# host copies), one download at the end.
RESIDENT = DRIVER.replace("local kz, e = Mara.advance(P, 0.0)",
                          "Mara.upload_primitive(P)\nlocal kz, e = Mara.advance_device(0.0)") \
                 .replace("kz, e = Mara.advance(P, dt)", "kz, e = Mara.advance_device(dt)") \
                 .replace("log:close()", "log:close()\nMara.download_primitive(P)")


@needs_host
@pytest.mark.gpu
def test_device_resident_loop_matches_the_reference(tmp_path):
    """Mara.upload_primitive / advance_device / download_primitive: the reference's driver loop
    without the per-step host round trips gives the reference's states, dt and error counts."""
    assert RESIDENT != DRIVER and "advance_device(dt)" in RESIDENT
    kw = dict(riemann="hlld", advance="rk2", extrap="plm")
    n = (12, 10, 8)
    P0 = ics.turbulence_box(n, seed=73, vrms=0.2)
    inp = tmp_path / "P0.bin"
    P0.astype(np.float64).tofile(inp)
    out = tmp_path / "P_res.bin"
    with LuaHost() as h:
        h.run(RESIDENT.format(inp=inp, out=out, steps=4, n0=n[0], n1=n[1], n2=n[2], **kw))
    Pg = np.fromfile(out).reshape(P0.shape)
    lg = open(str(out) + ".txt").read().split("\n")
    Pr, lr = _run_driver(tmp_path, "ref", kw, n, 4, P0)
    for a, b in zip(lg[:5], lr[:5]):
        ea, eb = a.split(), b.split()
        assert ea[0] == eb[0]
        if len(ea) > 1:
            assert abs(float(ea[1]) - float(eb[1])) <= 1e-12 * float(eb[1])
    assert np.abs(Pg - Pr).max() <= 1e-10 * np.abs(Pr).max()


# Every Mara.measure.* the reference's drivers log every few iterations, called as they call
# them (tables from mean_cons / mean_prim / mean_velocity, a keyed table from mean_energies,
# two numbers from the mean/extreme pairs), written one number per line.
MEASURES = r"""
local function put(log, x)
  if type(x) == 'table' then
    if #x > 0 then for i = 1, #x do log:write(string.format('%.17g\n', x[i])) end
    else for _, k in ipairs({'magnetic', 'kinetic', 'internal', 'total'}) do
      log:write(string.format('%.17g\n', x[k])) end end
  else log:write(string.format('%.17g\n', x)) end
end
local function measure_all(log)
  put(log, Mara.measure.mean_cons())
  put(log, Mara.measure.mean_prim())
  put(log, Mara.measure.mean_energies())
  put(log, Mara.measure.mean_velocity())
  local a, b = Mara.measure.mean_max_temperature(); put(log, a); put(log, b)
  a, b = Mara.measure.mean_max_magnetic_field(); put(log, a); put(log, b)
  a, b = Mara.measure.mean_max_sonic_mach(); put(log, a); put(log, b)
  a, b = Mara.measure.mean_min_alfvenic_mach(); put(log, a); put(log, b)
  put(log, Mara.measure.max_lorentz_factor())
  put(log, Mara.cooling_rate(0.1))
end
"""

# A crash ladder in the manner of the reference's driven-turbulence driver: on a failed step,
# switch to the CTU-Hancock operator with a smaller limiter, diffuse around the failed zones,
# halve dt and retry; the scheme goes back after a recovered step.
LADDER = MEASURES + r"""
Mara.start()
Mara.set_fluid('rmhd')
Mara.set_eos('gamma-law', 4.0 / 3.0)
Mara.set_godunov('plm-split')
Mara.set_boundary('periodic')
Mara.set_riemann('hllc')
Mara.set_advance('rk3')
Mara.config_solver({extrap='plm', theta=2.0}, true)
Mara.set_domain({0,0,0}, {1,1,1}, {12,12,12}, 8, 3)
local f = io.open('{inp}', 'rb'); local P = buffer.new_buffer(f:read('*a')); f:close()
local log = io.open('{out}.txt', 'w')
local kz, e = Mara.advance(P, 0.0)
for n = 1, 4 do
  local dt = Mara.get_timestep(0.3)
  kz, e = Mara.advance(P, dt)
  local attempt = 0
  while e ~= 0 and attempt < 3 do
    attempt = attempt + 1
    log:write(string.format('fail %d %d\n', n, e))
    Mara.set_godunov('plm-muscl')
    Mara.set_advance('single')
    Mara.config_solver({theta=1.5 - 0.25 * attempt}, true)
    Mara.diffuse(P, 0.2)
    dt = 0.5 * dt
    kz, e = Mara.advance(P, dt)
  end
  log:write(string.format('step %d %d %d %.17g\n', n, attempt, e, dt))
  if attempt > 0 then
    Mara.set_godunov('plm-split')
    Mara.set_advance('rk3')
    Mara.config_solver({theta=2.0}, true)
  end
end
measure_all(log)
log:close()
local g = io.open('{out}', 'wb'); g:write(tostring(P)); g:close()
Mara.close()
"""


def _run_script(tmp_path, which, script, P0, **fmt):
    inp = tmp_path / f"in_{which}.bin"
    P0.astype(np.float64).tofile(inp)
    out = tmp_path / f"out_{which}.bin"
    code = script.replace("{inp}", str(inp)).replace("{out}", str(out))
    for k, v in fmt.items():
        code = code.replace("{" + k + "}", str(v))
    if which == "gpu":
        with LuaHost() as h:
            h.run(code)
    else:
        from oracle import RefOracle, Scheme
        ref = RefOracle(Scheme(n=P0.shape[:3]))
        ref.dostring(code)
        ref.close()
    return np.fromfile(out).reshape(P0.shape), open(str(out) + ".txt").read().split("\n")


def _compare_measures(lg, lr, rel):
    a = np.array([float(x) for x in lg if x])
    b = np.array([float(x) for x in lr if x])
    assert a.shape == b.shape
    scale = np.maximum(np.abs(b), 1e-6 * np.abs(b).max())
    assert (np.abs(a - b) <= rel * scale).all(), np.abs(a - b) / scale


def test_crash_ladder_runs_in_the_reference(tmp_path):
    """The ladder script itself in the reference's interpreter: step 3 fails and is recovered
    by diffusion plus the CTU-Hancock fallback."""
    from ctf_b200 import ics
    P0 = ics.turbulence_box((12, 12, 12), seed=1)
    P, lines = _run_script(tmp_path, "ref", LADDER, P0)
    assert any(ln.startswith("fail 3") for ln in lines)
    steps = [ln.split() for ln in lines if ln.startswith("step")]
    assert len(steps) == 4 and all(s[3] == "0" for s in steps)
    assert np.isfinite(P).all()


@needs_host
@pytest.mark.gpu
def test_crash_ladder_matches_the_reference(tmp_path):
    """Mara.diffuse, in-place scheme changes (plm-split <-> plm-muscl, rk3 <-> single, theta)
    and every Mara.measure.* in both hosts: the same failures and recoveries, dt to 1e-12, the
    state to 1e-10, the measures of the last stage's primitives to 1e-9."""
    from ctf_b200 import ics
    P0 = ics.turbulence_box((12, 12, 12), seed=1)
    Pg, lg = _run_script(tmp_path, "gpu", LADDER, P0)
    Pr, lr = _run_script(tmp_path, "ref", LADDER, P0)
    ev_g = [ln for ln in lg if ln.startswith(("fail", "step"))]
    ev_r = [ln for ln in lr if ln.startswith(("fail", "step"))]
    assert len(ev_g) == len(ev_r) and any(ln.startswith("fail") for ln in ev_r)
    for a, b in zip(ev_g, ev_r):
        ea, eb = a.split(), b.split()
        assert ea[:4] == eb[:4], (a, b)
        if ea[0] == "step":
            assert abs(float(ea[4]) - float(eb[4])) <= 1e-12 * float(eb[4])
    assert np.abs(Pg - Pr).max() <= 1e-10 * np.abs(Pr).max()
    n_ev = len(ev_r)
    _compare_measures(lg[n_ev:], lr[n_ev:], 1e-9)


MEASURE_DRIVER = MEASURES + r"""
Mara.start()
Mara.set_fluid('rmhd')
Mara.set_eos('gamma-law', 4.0 / 3.0)
Mara.set_godunov('plm-split')
Mara.set_boundary('periodic')
Mara.set_riemann('hlld')
Mara.set_advance('rk2')
Mara.config_solver({extrap='plm', theta=2.0}, true)
Mara.set_domain({0,0,0}, {1,1,1}, {10,8,6}, 8, 3)
local f = io.open('{inp}', 'rb'); local P = buffer.new_buffer(f:read('*a')); f:close()
local log = io.open('{out}.txt', 'w')
Mara.set_primitive(P)
measure_all(log)
log:close()
local g = io.open('{out}', 'wb'); g:write(tostring(P)); g:close()
Mara.close()
"""


@needs_host
@pytest.mark.gpu
def test_measurement_block_matches_the_reference(tmp_path):
    """The measures of a given primitive array (Mara.set_primitive): extremes exactly, means
    to 1e-12 (relative to the value, or to a millionth of the largest measure for the signed
    means near zero)."""
    from ctf_b200 import ics
    P0 = ics.turbulence_box((10, 8, 6), seed=45, vrms=0.4)
    _, lg = _run_script(tmp_path, "gpu", MEASURE_DRIVER, P0)
    _, lr = _run_script(tmp_path, "ref", MEASURE_DRIVER, P0)
    _compare_measures(lg, lr, 1e-12)
