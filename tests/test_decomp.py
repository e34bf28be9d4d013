"""Domain decomposition host logic on the CPU: block geometry, the multiplicity tables of
the error counts, the slab layout, and the guard exchange schedule -- serial, and overlapped
with the core's c2p (the slabs must read only boundary-shell zones) -- across world_size-2
and -4 gloo process groups (CPU tensors), against the periodic guard fill of the whole box."""
import os

import numpy as np
import pytest

from ctf_b200 import decomp
from ctf_b200.decomp import NG, Layout


def test_blocks_partition_the_axis():
    for N in (12, 13, 64):
        for p in (1, 2, 3, 4):
            cover = []
            for c in range(p):
                off, n = decomp.block(N, p, c)
                cover += list(range(off, off + n))
            assert cover == list(range(N))


def test_rank_dims():
    assert decomp.rank_dims(1, 3, (64, 64, 64)) == (1, 1, 1)
    assert decomp.rank_dims(2, 3, (64, 64, 64)) == (2, 1, 1)
    assert decomp.rank_dims(8, 3, (64, 64, 64)) == (2, 2, 2)
    assert decomp.rank_dims(4, 2, (64, 32)) == (4, 1, 1) or decomp.rank_dims(4, 2, (64, 32)) == (2, 2, 1)
    d = decomp.rank_dims(6, 3, (96, 64, 64))
    assert d[0] * d[1] * d[2] == 6


@pytest.mark.parametrize("N,p", [(12, 1), (12, 2), (12, 3), (13, 4), (9, 3)])
def test_multiplicity_tables_count_every_guarded_copy(N, p):
    """Brute force: lay every block's guarded index range on the periodic axis and count."""
    count = np.zeros(N, dtype=int)
    for r in range(p):
        off, n = decomp.block(N, p, r)
        for q in range(n + 2 * NG):
            count[(off + q - NG) % N] += 1
    for c in range(p):
        off, n = decomp.block(N, p, c)
        assert list(decomp.multiplicity_table(N, p, c)) == list(count[off:off + n])
    if p == 1:   # one block: the zone and its own periodic images (the device's images_1d)
        assert count[0] == 2 and count[NG] == 1 and count[N - 1] == 2


def test_slab_pack_unpack_layout():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((10, 9, 8, 8))
    for d, n in ((0, 4), (1, 3), (2, 2)):
        for side in (0, 1):
            buf = decomp.pack_slab(A, d, side, n)
            assert buf.shape == (8, NG * (A.size // 8) // A.shape[d])
            B = np.zeros_like(A)
            decomp.unpack_slab(B, buf, d, side, n)
            first_src = NG if side == 0 else n
            first_dst = 0 if side == 0 else n + NG
            src = np.take(A, range(first_src, first_src + NG), axis=d)
            dst = np.take(B, range(first_dst, first_dst + NG), axis=d)
            assert np.array_equal(src, dst)
            # buffer order: [component][layer][cross-section in zone order]
            lay = np.moveaxis(src, d, 0)
            assert np.array_equal(buf[3].reshape(lay.shape[:3]), lay[..., 3])


def _global_field(N, seed=1):
    """A random global field with guards from the periodic fill of the whole box."""
    rng = np.random.default_rng(seed)
    G = tuple(v + 2 * NG for v in N) + (1,) * (3 - len(N))
    A = rng.standard_normal(G + (8,))
    for d in range(len(N)):
        decomp.periodic_fill(A, d, N[d])
    return A


def _worker(rank, world, port, N, dims, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        L = Layout(N=N, dims=dims, x0=(0.0,) * len(N), x1=(1.0,) * len(N))
        Ag = _global_field(N)
        _, off, n, _, _ = L.local(rank)
        sl = tuple(slice(off[d], off[d] + n[d] + 2 * NG) if d < len(N) else slice(None) for d in range(3))
        want = Ag[sl].copy()
        A = want.copy()
        # garbage in every guard layer, then the exchange schedule
        for d in range(len(N)):
            idx = [slice(None)] * 3
            idx[d] = list(range(NG)) + list(range(n[d] + NG, n[d] + 2 * NG))
            A[tuple(idx)] = np.nan
        decomp.exchange_numpy(A, L, rank, decomp.TorchTransport(dist))
        # the overlapped schedule: shells converted, slabs exchanged, cores converted
        B = decomp.overlapped_exchange_numpy(want, L, rank, decomp.TorchTransport(dist))
        # the error/MaxLambda reductions of an advance (sum of counters, max of bits)
        import torch
        errs = torch.tensor([0, rank + 1, 0, 0, 0], dtype=torch.int32)
        bits = torch.tensor([int(np.float64(0.5 + rank).view(np.int64))], dtype=torch.int64)
        tr = decomp.TorchTransport(dist)
        tr.sum_(errs)
        tr.max_(bits)
        q.put((rank, bool(np.array_equal(A, want)) and bool(np.array_equal(B, want)), errs.tolist(),
               float(bits.numpy().view(np.float64)[0])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("N,dims", [((12, 10, 8), (2, 1, 1)), ((12, 10, 8), (2, 2, 1)),
                                    ((16, 12), (2, 2, 1)), ((9, 8, 6), (1, 2, 2))])
def test_gloo_exchange_reproduces_the_periodic_fill(N, dims):
    import socket
    import torch.multiprocessing as mp
    world = dims[0] * dims[1] * dims[2]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, N, dims, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, errs, ml in res:
        assert ok, rank
        assert errs == [0, world * (world + 1) // 2, 0, 0, 0]
        assert ml == 0.5 + world - 1


def test_shell_mask_is_the_zones_within_ng_of_a_split_face():
    m = decomp.shell_mask((10, 8, 7), [0])
    assert m[:NG].all() and m[-NG:].all() and not m[NG:-NG].any()
    m = decomp.shell_mask((10, 8, 7), [1, 2])
    assert m[:, :NG].all() and m[:, :, -NG:].all() and not m[:, NG:-NG, NG:-NG].any()
    assert decomp.shell_mask((5, 8, 8), [0]).all()      # thinner than 2 Ng: all shell
