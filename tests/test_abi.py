"""The C-ABI library loads and exports every entry point include/mara_gpu.h declares
(CPU-only: no compute call needs a GPU here)."""
import ctypes
import os
import re

import pytest

from ctf_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            names += re.findall(r"^\s*(?:int|const char \*|void)\s+(mgpu_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "mgpu_advance" in names and "mgpu_create" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.build())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_default_config_is_the_reference_defaults():
    lib = _lib.load()
    c = _lib.MgpuConfig()
    assert lib.mgpu_default_config(ctypes.byref(c)) == 0
    assert c.gamma == 4.0 / 3.0 and c.theta == 2.0 and c.sz10A == 50.0 and c.pfloor == -1.0
    assert c.recon == 1 and c.riemann == 2 and c.rk == 2 and c.precision == 0


def test_bad_config_is_rejected_without_a_gpu():
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    c.rk = 7
    h = ctypes.c_void_p()
    assert lib.mgpu_create(ctypes.byref(c), ctypes.byref(h)) == 1   # MGPU_ERR_ARG
    assert not h.value


@pytest.mark.parametrize("field,value,code", [
    ("layout", 7, 1),                 # no such layout: MGPU_ERR_ARG
    ("godunov", 4, 1),                # no such integration scheme
    ("precision", 3, 1),
    ("riemann", 3, 1),
    ("recon", -1, 1),
    ("gamma", 1.0, 1),                # gamma-law index must exceed 1
])
def test_config_fields_are_checked_without_a_gpu(field, value, code):
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    setattr(c, field, value)
    h = ctypes.c_void_p()
    assert lib.mgpu_create(ctypes.byref(c), ctypes.byref(h)) == code
    assert not h.value


@pytest.mark.parametrize("field,value", [("rk", 4), ("godunov", 1)])
def test_lean_layout_limits_are_checked_without_a_gpu(field, value):
    """The lean layout runs 'plm-split' with single, rk2 or rk3: other schemes are
    MGPU_ERR_UNSUPPORTED before any device work."""
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    c.layout = 1                      # MGPU_LAYOUT_LEAN
    setattr(c, field, value)
    h = ctypes.c_void_p()
    assert lib.mgpu_create(ctypes.byref(c), ctypes.byref(h)) == 5
    assert not h.value


def test_null_handle_is_an_argument_error():
    lib = _lib.load()
    assert lib.mgpu_advance(None, 0.0, None) == 1
    assert lib.mgpu_destroy(None) == 0


def test_ensemble_create_rejects_bad_arguments_without_a_gpu():
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    N = (ctypes.c_int * 4)(16, 16, 2, 16)
    h = ctypes.c_void_p()
    create = lib.mgpu_ensemble_create
    assert create(ctypes.byref(c), 2, 2, N, None, None, ctypes.byref(h)) == 1     # N < 3 on an axis
    assert create(ctypes.byref(c), 4, 1, N, None, None, ctypes.byref(h)) == 1     # 4 dimensions
    assert create(ctypes.byref(c), 2, 0, N, None, None, ctypes.byref(h)) == 1     # no boxes
    c.learned_c2p = 1
    assert create(ctypes.byref(c), 2, 1, N, None, None, ctypes.byref(h)) == 5     # MGPU_ERR_UNSUPPORTED
    assert not h.value
    assert lib.mgpu_ensemble_advance(None, 1, 0, None, 0.0, 1) == 1
    assert lib.mgpu_ensemble_destroy(None) == 1


def test_ensemble_box_sizes_are_log_uniform():
    import numpy as np
    from ctf_b200.ensemble import kh_sizes
    sizes = kh_sizes(256, seed=0)
    sides = np.array([s[0] for s in sizes])
    assert len(sizes) == 256 and all(s[0] == s[1] for s in sizes)
    assert sides.min() >= 64 and sides.max() <= 512 and np.all(sides % 8 == 0)
    # log-uniform: the median side is near the geometric mean sqrt(64 * 512) = 181
    assert 150 <= np.median(sides) <= 215
    assert kh_sizes(256, seed=0) == sizes


def _noalloc_call(lib, cfg, n, errbuf, nd=None, src=16, dst=16, x0=True):
    """mgpu_advance_noalloc with placeholder device pointers: every argument check returns
    before the call touches the device, so this runs without a GPU."""
    nd = len(n) if nd is None else nd
    m = max(nd, 1)
    X0 = (ctypes.c_double * m)(*([0.0] * m)) if x0 else None
    X1 = (ctypes.c_double * m)(*([1.0] * m))
    N = (ctypes.c_int * m)(*(list(n) + [8] * m)[:m])
    err, ml = ctypes.c_int(-1), ctypes.c_double(0.0)
    return lib.mgpu_advance_noalloc(ctypes.byref(cfg), X0, X1, N, nd, ctypes.c_void_p(src),
                                    ctypes.c_void_p(dst), ctypes.c_double(1e-3), ctypes.byref(err),
                                    ctypes.byref(ml), None, errbuf, len(errbuf))


@pytest.mark.parametrize("field,value,msg", [
    ("precision", 1, "needs an rmhd FP64 plm-split configuration"),
    ("learned_c2p", 1, "needs an rmhd FP64 plm-split configuration"),
    ("godunov", 1, "needs an rmhd FP64 plm-split configuration"),
    ("layout", 1, "needs an rmhd FP64 plm-split configuration"),
    ("rk", 5, "needs an rmhd FP64 plm-split configuration"),
    ("gamma", 1.0, "needs an rmhd FP64 plm-split configuration"),
])
def test_noalloc_config_checks_without_a_gpu(field, value, msg):
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    setattr(c, field, value)
    buf = ctypes.create_string_buffer(256)
    assert _noalloc_call(lib, c, (8, 8, 8), buf) == 1      # MGPU_ERR_ARG
    assert msg in buf.value.decode()


@pytest.mark.parametrize("case,msg", [
    ("nd0", "1, 2 or 3 dimensions"),
    ("nd4", "1, 2 or 3 dimensions"),
    ("small_axis", "needs N >= 3 on every axis"),
    ("too_many_zones", "more than the 11520"),
    ("null_input", "null argument"),
    ("null_output", "null argument"),
    ("null_extent", "null argument"),
])
def test_noalloc_domain_checks_without_a_gpu(case, msg):
    lib = _lib.load()
    c = _lib.MgpuConfig()
    lib.mgpu_default_config(ctypes.byref(c))
    buf = ctypes.create_string_buffer(256)
    kw = {}
    n = (8, 8, 8)
    if case == "nd0":
        kw["nd"] = 0
    elif case == "nd4":
        n, kw["nd"] = (8, 8, 8, 8), 4
    elif case == "small_axis":
        n = (8, 2, 8)
    elif case == "too_many_zones":
        n = (20, 20, 20)
    elif case == "null_input":
        kw["src"] = None
    elif case == "null_output":
        kw["dst"] = None
    else:
        kw["x0"] = False
    assert _noalloc_call(lib, c, n, buf, **kw) == 1
    assert msg in buf.value.decode()
