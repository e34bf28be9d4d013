"""Host transfers of large pageable buffers (include/mara_gpu.h: mgpu_upload_prim,
mgpu_download_prim, mgpu_advance_host).

From 64 MB on, a buffer that is not pinned goes through the solver's pinned staging copy, with
the host copies on a pool of threads, chunk by chunk.  Uploads, downloads and a whole
Mara.advance(buf, dt) through a pageable buffer give the same bytes as through a pinned one.
"""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu

N = (160, 160, 160)   # 166^3 guarded zones: 292 MB of AoS primitives, two staging chunks


def _pinned_like(P):
    import torch
    t = torch.empty(P.size, dtype=torch.float64, pin_memory=True)
    a = t.numpy().reshape(P.shape)
    a[...] = P
    return t, a


@pytest.mark.parametrize("layout,precision", [("standard", "fp64"), ("lean", "fp32")])
def test_pageable_transfers_match_pinned(layout, precision):
    P0 = ics.turbulence_box(N, seed=5, vrms=0.2)
    kw = dict(extrap="plm", riemann="hlld", advance="rk2", precision=precision, layout=layout)
    a, b = Solver(Scheme(**kw), N), Solver(Scheme(**kw), N)
    keep, pinned = _pinned_like(P0)
    keep_out, pinned_out = _pinned_like(np.zeros_like(P0))
    a.upload(P0.copy())            # pageable: staged
    b.upload(pinned)               # pinned: direct
    assert np.array_equal(a.download(), b.download(pinned_out))
    assert a.advance(0.0) == 0 and b.advance(0.0) == 0
    dt = a.get_timestep(0.3)
    if layout == "lean":           # the unpipelined call, so that the transfers themselves run
        a.set_pipeline(0)
        b.set_pipeline(0)
    pageable = P0.copy()
    _, ea = a.advance_host(pageable, dt)
    _, eb = b.advance_host(pinned, dt)
    assert ea == eb == 0
    assert np.array_equal(pageable, pinned)
    del keep, keep_out


def test_pageable_range_transfers_match_pinned():
    """Ranges that start and end inside the array (mgpu_upload_prim_range,
    mgpu_download_prim_range): the staged chunks follow the range's first zone."""
    from ctf_b200.mara import _dp
    P0 = ics.turbulence_box(N, seed=9, vrms=0.2)
    a, b = Solver(Scheme(), N), Solver(Scheme(), N)   # FP64, standard layout
    flat = P0.reshape(-1, 8)
    z0 = 100_003
    cnt = flat.shape[0] - z0 - 7                      # 4.47 M zones (286 MB): two chunks
    R = flat[z0:z0 + cnt].copy()
    R[:, 0] *= 1.01                                   # a density change, still physical
    for s in (a, b):
        s.upload(P0.copy())
    a.upload_range(R.copy(), z0)                      # pageable: staged
    keep, pinned = _pinned_like(R)
    b.upload_range(pinned, z0)                        # pinned: direct
    assert np.array_equal(a.download(), b.download())
    keep_out, pinned_out = _pinned_like(np.zeros_like(R))
    assert b.lib.mgpu_download_prim_range(b.h, _dp(pinned_out), z0, cnt) == 0
    got = a.download_range(z0, cnt)                   # pageable: staged
    assert np.array_equal(got, pinned_out) and np.array_equal(got, R)
    del keep, keep_out
