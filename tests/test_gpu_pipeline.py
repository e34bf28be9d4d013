"""The pipelined Mara.advance(buf, dt) of the lean layout (mgpu_advance_host over slabs of x
rows, include/mara_gpu.h) against the same call unpipelined (mgpu_set_pipeline(h, 0)).

Every window launch computes exactly the faces and zones of the whole-box launch that fall in
its slab, so the caller's buffer, the error count, MaxLambda and the zone c2p statistics are
the same bit for bit, in FP32 bulk (with and without the learned c2p) and FP64, for pinned
buffers (copies out overlap the advance) and pageable ones (copied out after the commit).
A failing advance leaves a pinned buffer exactly as it was, as luaC_Mara_advance does
(Mara/mara.cpp:325-334), although its copies out had started.
"""
import ast

import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu

ZONE_STATS = ("c2p_calls", "c2p_iters", "c2p_attempt", "c2p_failed", "errors", "committed")


class _Pinned(np.ndarray):
    pass


def _buf(P, pinned):
    if not pinned:
        return P.copy()
    import torch
    t = torch.empty(P.size, dtype=torch.float64, pin_memory=True)
    a = t.numpy().reshape(P.shape).view(_Pinned)
    a[...] = P
    a.storage_owner = t
    return a


def _run(P0, n, slabs, dts, pinned, precision="fp32", learned=False, **kw):
    scheme = Scheme(precision=precision, layout="lean", learned_c2p=learned, **kw)
    s = Solver(scheme, n)
    if learned:
        from ctf_b200 import train_c2p
        s.set_c2p_network(train_c2p.load())
    s.set_pipeline(slabs)
    buf = _buf(P0, pinned)
    out = []
    for dt in dts:
        _, e = s.advance_host(buf, float(dt))
        st = s.stats()
        out.append((e, np.array(buf), s.get_timestep(0.3), {k: st[k] for k in ZONE_STATS}, s.pipeline()[1]))
    return out


def _dts(P0, n, **kw):
    ref = Solver(Scheme(**kw), n)
    ref.upload(P0.copy())
    assert ref.advance(0.0) == 0
    return [ref.get_timestep(0.3)] * 3


def _same(a, b, slabs):
    for k, ((ea, Pa, dta, sa, la), (eb, Pb, dtb, sb, lb)) in enumerate(zip(a, b)):
        assert la == 0 and lb == slabs, (k, la, lb)
        assert ea == eb, k
        assert np.array_equal(Pa, Pb), (k, np.abs(Pa - Pb).max())
        assert dta == dtb, k
        assert sa == sb, (k, sa, sb)


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("slabs", [3, 6])
def test_pipelined_fp32_is_the_unpipelined_call(slabs, pinned):
    n = (24, 20, 16)
    kw = dict(extrap="plm", riemann="hlld", advance="rk3")
    P0 = ics.turbulence_box(n, seed=17, vrms=0.3)
    dts = _dts(P0, n, **kw)
    _same(_run(P0, n, 0, dts, pinned, **kw), _run(P0, n, slabs, dts, pinned, **kw), slabs)


@pytest.mark.parametrize("advance", ["single", "rk2"])
def test_pipelined_weno5_four_row_slabs(advance):
    """Slabs of four rows: WENO5's stencil reaches three rows into each neighbour."""
    n = (24, 12, 20)
    kw = dict(extrap="weno5", riemann="hlld", advance=advance)
    P0 = ics.turbulence_box(n, seed=23, vrms=0.3)
    dts = _dts(P0, n, **kw)
    _same(_run(P0, n, 0, dts, True, **kw), _run(P0, n, 6, dts, True, **kw), 6)


def test_pipelined_fp64_and_learned():
    n = (16, 16, 16)
    kw = dict(extrap="plm", riemann="hlld", advance="rk3")
    P0 = ics.turbulence_box(n, seed=29, vrms=0.3)
    dts = _dts(P0, n, **kw)
    _same(_run(P0, n, 0, dts, True, "fp64", **kw), _run(P0, n, 4, dts, True, "fp64", **kw), 4)
    _same(_run(P0, n, 0, dts, True, "fp32", True, **kw), _run(P0, n, 4, dts, True, "fp32", True, **kw), 4)


@pytest.mark.parametrize("learned", [False, True])
def test_pipelined_stress_box_with_emergency_reset(learned):
    """The stress box with the emergency reset: zones fail and are reset in every step, a path
    that amplifies any difference in the last bits, and the state is still the same bit for
    bit."""
    n = (16, 16, 16)
    kw = dict(extrap="plm", riemann="hlld", advance="rk3", ereset=True, preset=0.01, dreset=1.0)
    P0 = ics.stress_box(n, seed=0)
    dts = _dts(P0, n, **kw)
    a = _run(P0, n, 0, dts, True, "fp32", learned, **kw)
    _same(a, _run(P0, n, 4, dts, True, "fp32", learned, **kw), 4)
    assert a[0][3]["c2p_failed"] > 0


def test_automatic_uneven_slabs():
    """From 96 x rows the automatic layout mixes 6-row and 16-row slabs (12 at 96 rows)."""
    n = (96, 12, 10)
    kw = dict(extrap="plm", riemann="hlld", advance="rk3")
    P0 = ics.turbulence_box(n, seed=37, vrms=0.3)
    dts = _dts(P0, n, **kw)
    _same(_run(P0, n, 0, dts, True, **kw), _run(P0, n, -1, dts, True, **kw), 12)


def test_default_pipeline_and_standard_layout():
    n = (16, 16, 16)
    P0 = ics.turbulence_box(n, seed=3, vrms=0.2)
    s = Solver(Scheme(precision="fp32", layout="lean"), n)
    assert s.pipeline() == (-1, 0)
    buf = _buf(P0, True)
    s.advance_host(buf, 1e-3)
    assert s.pipeline() == (-1, 3)        # automatic: at least three slabs
    t = Solver(Scheme(precision="fp32"), n)
    t.advance_host(P0.copy(), 1e-3)
    assert t.pipeline()[1] == 0           # the standard layout is not pipelined
    with pytest.raises(Exception):
        s.set_pipeline(2)


@pytest.mark.parametrize("pinned", [True, False])
def test_failing_advance_leaves_the_buffer(golden, pinned):
    """The reference's failing HLLC step (4 failed zones): the same count as unpipelined, the
    caller's buffer unchanged although its copies out had started, and a smaller step then
    commits to the same state as the unpipelined solver's."""
    g = golden("step_hllc_fail_12.npz")
    kw = ast.literal_eval(str(g["scheme"]))
    n = kw.pop("n")
    before = np.ascontiguousarray(g["states"][1])
    dt = float(g["dts"][2])
    runs = {}
    for slabs in (0, 3):
        s = Solver(Scheme(precision="fp64", layout="lean", **kw), n)
        s.set_pipeline(slabs)
        buf = _buf(before, pinned)
        _, e = s.advance_host(buf, dt)
        assert e == g["errors"][3] and e > 0
        assert s.pipeline()[1] == slabs
        assert np.array_equal(np.array(buf), before)
        _, e2 = s.advance_host(buf, 0.25 * dt)
        assert e2 == 0
        runs[slabs] = np.array(buf)
    assert np.array_equal(runs[0], runs[3])
