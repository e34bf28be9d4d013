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
        ok, msg = pcall(Mara.diffuse)
        assert(not ok and msg:find('diffuse is not provided'))
        ok, msg = pcall(Mara.measure.mean_cons)
        assert(not ok and msg:find('mean_cons is not provided'))
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
