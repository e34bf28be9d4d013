"""The allocation-free entry point, mgpu_advance_noalloc, through the C ABI.

It serves callers that may not allocate device memory (allocation-free sections of a larger
application, real-time loops, hosts that only hand out buffers they already own): it keeps
its working arrays in a fixed region of the library's own device memory.  Its result must
match the regular entry point's (mgpu_create / mgpu_set_domain / mgpu_advance), within the
parity tolerance of the other GPU tests, on two calls in a row -- the second call reuses a
region that still holds the first call's contents.

This file is collected last on purpose, and must pass both alone in a fresh process and
after the other tests.
"""
import ctypes

import numpy as np
import pytest

from ctf_b200 import _lib, ics
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10   # the plain-FP64 parity bound used by tests/test_gpu_parity.py


def _rel_linf(a, b):
    a, b = a.reshape(-1, 8), b.reshape(-1, 8)
    out = 0.0
    for q in range(8):
        s = np.abs(b[:, q]).max()
        out = max(out, np.abs(a[:, q] - b[:, q]).max() / (s if s > 0 else 1.0))
    return out


def _noalloc(lib, cfg, n, src, dst, dt):
    nd = len(n)
    x0 = (ctypes.c_double * nd)(*([0.0] * nd))
    x1 = (ctypes.c_double * nd)(*([1.0] * nd))
    N = (ctypes.c_int * nd)(*n)
    err, ml = ctypes.c_int(-1), ctypes.c_double(0.0)
    msg = ctypes.create_string_buffer(256)
    rc = lib.mgpu_advance_noalloc(ctypes.byref(cfg), x0, x1, N, nd, ctypes.c_void_p(src),
                                  ctypes.c_void_p(dst), ctypes.c_double(dt), ctypes.byref(err),
                                  ctypes.byref(ml), None, msg, len(msg))
    return rc, err.value, ml.value, msg.value.decode()


@pytest.mark.parametrize("scheme_kw,n", [
    (dict(extrap="plm", riemann="hlld", advance="rk2"), (10, 12, 14)),
    (dict(extrap="weno5", riemann="hllc", advance="rk3"), (40, 36)),
    (dict(extrap="plm", riemann="hll", advance="rk4"), (9, 8, 11)),     # the K registers
    (dict(extrap="weno5", riemann="hlld", advance="single"), (200,)),   # a 1D box
])
def test_noalloc_matches_regular_entry_point_twice(scheme_kw, n):
    import torch
    torch.cuda.set_device(0)
    lib = _lib.load()
    scheme = Scheme(**scheme_kw)
    cfg = scheme.to_config()
    if len(n) == 3:
        P0 = ics.turbulence_box(n, seed=21)
    elif len(n) == 2:
        P0 = ics.kh_box(n, seed=21)
    else:   # a line across the layers of a 2D shear box, laid along x: a 1D state whose
        # density, velocity and field all vary
        P0 = np.ascontiguousarray(ics.kh_box((8, n[0]), seed=21)[5].reshape(n[0] + 6, 1, 1, 8))

    ref = Solver(scheme, n)
    ref.upload(P0.copy())
    assert ref.advance(0.0) == 0
    dt = ref.get_timestep(0.3)
    ref.upload(P0.copy())

    d_in = torch.tensor(P0, device="cuda")
    d_mid = torch.zeros_like(d_in)
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    free_before = None
    for src, dst in ((d_in, d_mid), (d_mid, d_out)):
        assert ref.advance(dt) == 0
        rc, errors, ml, msg = _noalloc(lib, cfg, n, src.data_ptr(), dst.data_ptr(), dt)
        torch.cuda.synchronize()
        assert rc == 0, msg
        assert errors == 0
        assert abs(ml - ref.max_lambda) <= 1e-12 * ref.max_lambda
        got = dst.cpu().numpy()
        assert _rel_linf(got, ref.download()) <= STEP_TOL
        # the property that defines this entry point: after the first call (which may load
        # the library's device code), a call takes no device memory
        free = torch.cuda.mem_get_info()[0]
        if free_before is not None:
            assert free == free_before, (free_before, free)
        free_before = free


def test_noalloc_rejects_boxes_beyond_its_limit():
    import torch
    torch.cuda.set_device(0)
    lib = _lib.load()
    cfg = Scheme().to_config()
    n = (20, 20, 20)   # 26^3 = 17,576 guarded zones > MGPU_NOALLOC_MAX_ZONES
    buf = torch.zeros(26 ** 3 * 8, dtype=torch.float64, device="cuda")
    rc, _, _, msg = _noalloc(lib, cfg, n, buf.data_ptr(), buf.data_ptr(), 1e-3)
    assert rc == 1 and "more than the 11520" in msg
