"""The issue order of the pipelined host advance (mgpu_pipeline_schedule), checked on the CPU
against a model of what each operation reads and writes.

The model tracks, per interior x row, which stage's primitives each of the two stage arrays
holds (stage v lives in array (v + K) % 2, so the closing c2p's in the solver's own) and which
stage's sum the Runge-Kutta register holds.  Each operation asserts that every row it reads
holds the version it needs -- not yet written (a read before the producer) and already
overwritten (a write before the last reader) both fail -- and then writes its own rows.
Rows of primitives are periodic in x (the end slabs' guard images are their neighbours'
rows).  A sweep reads the stage primitives up to three rows beyond its slab (WENO5).  CT reads
the y and z face fields one row beyond its slab: the same operation's sweeps compute those halo
rows, except the one next to the neighbour toward slab 0, whose sweeps computed it as their own
row (face fields have no periodic images: rows -1 and n0 are guard rows of their own).
"""
import ctypes

import numpy as np
import pytest

from ctf_b200 import _lib

REACH = 3   # rows of stage primitives a sweep reads beyond its slab


def schedule(S, K):
    lib = _lib.load()
    n = lib.mgpu_pipeline_schedule(S, K, None, 0)
    assert n > 0
    out = (ctypes.c_int * (2 * n))()
    assert lib.mgpu_pipeline_schedule(S, K, out, 2 * n) == n
    return [(out[2 * i], out[2 * i + 1]) for i in range(n)]


def bounds(n0, slabs=-1):
    lib = _lib.load()
    S = lib.mgpu_pipeline_bounds(n0, slabs, None, 0)
    if S == 0:
        return []
    out = (ctypes.c_int * (S + 1))()
    assert lib.mgpu_pipeline_bounds(n0, slabs, out, S + 1) == S
    return list(out)


def simulate(S, K, n0, wb=None):
    """Runs the schedule against the row model; returns the order the slabs finished in."""
    E = 2 * K + 2
    wb = wb or [n0 * s // S for s in range(S + 1)]
    pa = np.full((2, n0), -1)  # stage of the primitives in each stage array (-1: none yet)
    reg = np.full(n0, -1)      # last stage whose sweeps were added into the register
    finished = []

    def rows(s, ext=0):
        return np.arange(wb[s] - ext, wb[s + 1] + ext) % n0

    def arr(v):
        return pa[(v + K) % 2]

    for s, e in schedule(S, K):
        own = rows(s)
        if e == 0:                                  # upload: the committed primitives
            arr(0)[own] = 0
        elif e == E - 1:                            # download of the result
            assert (arr(K)[own] == K).all() and (reg[own] == K - 1).all(), (s, e)
            finished.append(s)
        elif e % 2 == 1:                            # stage k's sweeps + CT
            k = (e - 1) // 2
            assert (arr(k)[rows(s, REACH)] == k).all(), (s, e)
            assert (reg[own] == k - 1).all(), (s, e)
            reg[own] = k
        else:                                       # stage k's c2p (k = K: the closing one)
            k = e // 2
            assert (reg[own] == k - 1).all(), (s, e)
            assert (arr(k - 1)[own] == k - 1).all(), (s, e)  # the previous primitives seed the ladder
            arr(k)[own] = k
    assert (arr(K) == K).all() and (reg == K - 1).all()
    return finished


def pred(S, s):
    """The neighbour whose same-stage sweeps computed one of this slab's halo rows."""
    if 1 <= s <= S // 2:
        return s - 1
    if S // 2 < s <= S - 2:
        return s + 1
    return None


def dependencies(S, K, s, e):
    """The operations that (s, e) waits for: the slab's previous one; for sweeps (odd e below
    the download) the neighbours' previous ones and the sweeps of pred(s)."""
    E = 2 * K + 2
    if e == 0:
        return []
    deps = [(s, e - 1)]
    if e % 2 == 1 and e != E - 1:
        deps += [((s - 1) % S, e - 1), ((s + 1) % S, e - 1)]
        if pred(S, s) is not None:
            deps.append((pred(S, s), e))
    return deps


def check_dag(S, K, n0, wb=None):
    """Every hazard ordered by the dependency graph alone, not only by the issue order (so the
    operations could also run on several streams): a read's producer and a write's previous
    writer and readers are ancestors.  Face fields: a sweep operation writes its own rows and
    the halo rows it computes, then CT reads its rows and one halo row each side; two writers
    of the same stage's face fields write the same values."""
    E = 2 * K + 2
    wb = wb or [n0 * s // S for s in range(S + 1)]
    anc = {}
    for op in schedule(S, K):
        a = set()
        for d in dependencies(S, K, *op):
            assert d in anc, (op, d)          # issued before its dependencies would deadlock
            a |= anc[d] | {d}
        anc[op] = a
    # per (array, row): [version, writers of that version, readers]
    state = {}

    def rows(s, ext=0):
        return [r % n0 for r in range(wb[s] - ext, wb[s + 1] + ext)]

    def face_rows(s):
        """Rows of y/z face fields this slab's sweeps write (unwrapped: -1 and n0 are guards)."""
        lo, hi = wb[s] - 1, wb[s + 1] + 1
        p = pred(S, s)
        if p == s - 1:
            lo += 1
        elif p == s + 1:
            hi -= 1
        return list(range(lo, hi))

    def done_before(x, op):
        return x == op or x in anc[op]

    def read(op, arr, rs, version):
        for r in rs:
            v, writers, readers = state[(arr, r)]
            assert v == version, (op, arr, r, v, version)
            assert any(done_before(w, op) for w in writers), (op, arr, r, writers)
            readers.add(op)

    def write(op, arr, rs, version, same_value_ok=False):
        for r in rs:
            old = state.get((arr, r))
            if old is not None:
                v, writers, readers = old
                if same_value_ok and v == version:            # the same stage's face fields
                    writers.add(op)
                    continue
                assert all(done_before(w, op) for w in writers), (op, arr, r, writers)
                assert all(done_before(x, op) for x in readers), (op, arr, r)
            state[(arr, r)] = [version, {op}, set()]

    def pa(v):
        return "pa%d" % ((v + K) % 2)

    for op in schedule(S, K):
        s, e = op
        own = rows(s)
        if e == 0:
            write(op, pa(0), own, 0)
            write(op, "u0", own, 0)
        elif e == E - 1:
            read(op, pa(K), own, K)
            read(op, "u1", own, K - 1)
        elif e % 2 == 1:
            k = (e - 1) // 2
            read(op, pa(k), rows(s, REACH), k)
            read(op, "u0", own, 0)
            if k > 0:
                read(op, "u1", own, k - 1)
            write(op, "u1", own, k)
            write(op, "bf", face_rows(s), k, same_value_ok=True)
            read(op, "bf", list(range(wb[s] - 1, wb[s + 1] + 1)), k)
        else:
            k = e // 2
            read(op, "u1", own, k - 1)
            read(op, pa(k - 1), own, k - 1)
            write(op, pa(k), own, k)


@pytest.mark.parametrize("n0", [12, 16, 24, 95, 96, 128, 256, 512, 1024])
def test_automatic_slabs(n0):
    """The automatic slabs cover the rows, at least 4 each, at least 3 of them; from 96 rows
    thin ones lie around slab 0 and around the far side; and every hazard is ordered."""
    wb = bounds(n0)
    S = len(wb) - 1
    assert S >= 3 and wb[0] == 0 and wb[-1] == n0
    w = np.diff(wb)
    assert (w >= 4).all()
    if n0 >= 96:
        assert w[0] == w[1] == w[-1] == 6 and w[S // 2] == 6 and w.max() >= 16
    for K in (1, 2, 3):
        assert sorted(simulate(S, K, n0, wb)) == list(range(S))
        check_dag(S, K, n0, wb)


def test_fixed_slabs_are_equal():
    assert bounds(512, 46) == [512 * s // 46 for s in range(47)]
    assert bounds(11) == [] and bounds(512, 200) == [512 * s // 128 for s in range(129)]
    lib = _lib.load()
    assert lib.mgpu_pipeline_bounds(512, 2, None, 0) < 0 and lib.mgpu_pipeline_bounds(512, 0, None, 0) < 0


@pytest.mark.parametrize("K", [1, 2, 3])
@pytest.mark.parametrize("S", [3, 4, 5, 7, 8, 16, 33])
def test_dependencies_order_every_hazard(S, K):
    for n0 in (4 * S, 4 * S + 3):
        check_dag(S, K, n0)


@pytest.mark.parametrize("K", [1, 2, 3])
@pytest.mark.parametrize("S", [3, 4, 5, 7, 8, 16, 33])
def test_schedule_respects_every_read(S, K):
    for n0 in (4 * S, 4 * S + 3, 32 * S):
        finished = simulate(S, K, n0)
        assert sorted(finished) == list(range(S))


@pytest.mark.parametrize("S,K", [(3, 3), (16, 3), (9, 2)])
def test_schedule_shape(S, K):
    """Every operation once, in order per slab; uploads outward from slab 0; the first
    downloads come before the last uploads when there are enough slabs to overlap them."""
    sched = schedule(S, K)
    E = 2 * K + 2
    assert len(sched) == S * E
    per = {s: [e for t, e in sched if t == s] for s in range(S)}
    assert all(per[s] == list(range(E)) for s in range(S))
    ups = [s for s, e in sched if e == 0]
    ring = [0] + [x for d in range(1, S) for x in (d, S - d)]
    assert ups == list(dict.fromkeys(ring))[:S]
    if S >= 16:
        first_dl = next(i for i, (s, e) in enumerate(sched) if e == E - 1)
        last_up = max(i for i, (s, e) in enumerate(sched) if e == 0)
        assert first_dl < last_up


def test_schedule_arguments_are_checked():
    lib = _lib.load()
    assert lib.mgpu_pipeline_schedule(2, 3, None, 0) < 0
    assert lib.mgpu_pipeline_schedule(4, 0, None, 0) < 0
    assert lib.mgpu_pipeline_schedule(4, 4, None, 0) < 0
    out = (ctypes.c_int * 4)()
    assert lib.mgpu_pipeline_schedule(4, 3, out, 4) < 0      # too small for 32 pairs


def test_pipeline_setting_needs_a_handle():
    lib = _lib.load()
    assert lib.mgpu_set_pipeline(None, -1) == 1
    assert lib.mgpu_get_pipeline(None, None, None) == 1
