"""Block domain decomposition of the periodic box over ranks (one GPU per rank).

The reference decomposes with MPI (DecomposedCartesianDomain, Mara/subgrids.cpp:12-147):
every rank holds its block with Ng guard layers, `Synchronize` exchanges the guard layers
dimension by dimension (x, then y, then z, each over the full guarded cross-section, so
edges and corners arrive through the sequence), ConsToPrim counts failures over every
guarded zone of every rank and sums the counts (Mara/hydro.cpp:201), and get_timestep takes
the minimum dt over ranks (Mara/mara_mpi.c:96-130).

Here a rank is one `mara.Solver` of its block.  `DecomposedSolver` drives its advance phase
by phase (`mgpu_advance_phase`), exchanging the stage primitives' guard slabs between the
c2p and the flux sweeps of every RK stage and reducing the error counters and MaxLambda
before the commit; all of it stays on the device streams (no host synchronisation per step).
The exchange overlaps the stage c2p: the boundary shell (zones within Ng of a split face,
all the slabs read) converts first, the slabs travel on a side stream while the core
converts, and the sweeps wait for both.
Two transports move the slabs:

* `TorchTransport` -- torch.distributed point-to-point (NCCL between GPUs; gloo on CPU
  tensors for the host-side tests), one process per rank;
* `LocalTransport` -- several ranks' solvers in one process on one device, slabs copied
  directly (for testing the decomposition on a single GPU; nothing waits on another rank).

The geometry helpers (`rank_dims`, `block`, `multiplicity_table`) and a numpy model of the
slab layout (`pack_slab`, `unpack_slab`, the same [component][layer][cross-section] order
as the device kernels) are plain Python so the schedule is testable without a GPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

NG = 3


# ---- geometry -----------------------------------------------------------------------------

def rank_dims(nranks: int, nd: int, N) -> tuple:
    """Ranks per dimension: a balanced factorisation (as MPI_Dims_create), larger factors on
    the dimensions with more zones; unused dimensions get 1."""
    dims = [1] * 3
    left = nranks
    f = 2
    factors = []
    while left > 1:
        while left % f == 0:
            factors.append(f)
            left //= f
        f += 1
    for p in sorted(factors, reverse=True):
        # give the factor to the used dimension with the most zones per rank
        d = max(range(nd), key=lambda k: N[k] / dims[k])
        dims[d] *= p
    return tuple(dims)


def block(N: int, p: int, c: int) -> tuple:
    """(offset, size) of block c of p along a dimension of N zones (remainder to the first)."""
    base, rem = divmod(N, p)
    size = base + (1 if c < rem else 0)
    off = c * base + min(c, rem)
    return off, size


def coords_of(rank: int, dims) -> tuple:
    """Rank -> block coordinates, x slowest (row-major, as MPI_Cart_create's default)."""
    cz = rank % dims[2]
    cy = (rank // dims[2]) % dims[1]
    cx = rank // (dims[1] * dims[2])
    return cx, cy, cz


def rank_of(coords, dims) -> int:
    return (coords[0] * dims[1] + coords[1]) * dims[2] + coords[2]


def multiplicity_table(N: int, p: int, c: int, ng: int = NG) -> np.ndarray:
    """For each interior index m of block c: how many guarded arrays of the p blocks along
    the dimension hold global zone off_c + m (guards wrap periodically)."""
    off, n = block(N, p, c)
    count = np.zeros(n, dtype=np.int32)
    for r in range(p):
        o, nr = block(N, p, r)
        glob = (o + np.arange(nr + 2 * ng) - ng) % N
        for g in glob:
            m = g - off
            if 0 <= m < n:
                count[m] += 1
    return count


# ---- numpy model of the slab layout (matches k_halo_copy) --------------------------------

def slab_index(shape, dim: int, first: int, ng: int = NG):
    """Zone indices (into a guarded array of `shape` = G0, G1, G2) of layers
    first..first+ng of `dim` over the full cross-section, in buffer order [layer][cross]."""
    sl = [slice(None)] * 3
    sl[dim] = slice(first, first + ng)
    return tuple(sl)


def pack_slab(A: np.ndarray, dim: int, side: int, n: int, ng: int = NG) -> np.ndarray:
    """A: guarded array (G0, G1, G2, ncomp).  side 0: interior layers [ng, 2ng); side 1:
    [n, n + ng).  Returns the buffer [comp][layer][cross]."""
    first = ng if side == 0 else n
    s = np.moveaxis(A[slab_index(A.shape[:3], dim, first, ng)], dim, 0)   # (ng, crossA, crossB, q)
    return np.ascontiguousarray(np.moveaxis(s, 3, 0)).reshape(A.shape[3], -1)


def unpack_slab(A: np.ndarray, buf: np.ndarray, dim: int, side: int, n: int, ng: int = NG):
    """Inverse of pack_slab into the guard layers: side 0 -> [0, ng), side 1 -> [n+ng, n+2ng)."""
    first = 0 if side == 0 else n + ng
    view = A[slab_index(A.shape[:3], dim, first, ng)]
    shp = np.moveaxis(view, dim, 0).shape            # (ng, crossA, crossB, q)
    s = buf.reshape((A.shape[3], shp[0], shp[1], shp[2]))
    A[slab_index(A.shape[:3], dim, first, ng)] = np.moveaxis(np.moveaxis(s, 0, 3), 0, dim)


def shell_mask(n, split, ng: int = NG) -> np.ndarray:
    """Interior zones of a block (n per dimension, 3 entries) within ng of a face of a split
    dimension: the zones the overlapped schedule converts before the exchange (the device's
    in_shell)."""
    idx = np.meshgrid(*[np.arange(m) for m in n], indexing="ij")
    mask = np.zeros(tuple(n), dtype=bool)
    for d in split:
        mask |= (idx[d] < ng) | (idx[d] >= n[d] - ng)
    return mask


def periodic_fill(A: np.ndarray, dim: int, n: int, ng: int = NG):
    """Guard layers of `dim` from the block's own opposite interior layers."""
    unpack_slab(A, pack_slab(A, dim, 1, n, ng), dim, 0, n, ng)
    unpack_slab(A, pack_slab(A, dim, 0, n, ng), dim, 1, n, ng)


# ---- transports ---------------------------------------------------------------------------

class TorchTransport:
    """Slabs through torch.distributed point-to-point; reductions with all_reduce.  Works
    with NCCL on CUDA tensors and with gloo on CPU tensors."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group

    def exchange(self, send_lo, send_hi, recv_lo, recv_hi, low: int, high: int):
        """send_lo -> low neighbour's high guards, send_hi -> high neighbour's low guards;
        recv_lo <- low neighbour's send_hi, recv_hi <- high neighbour's send_lo.  Every rank
        issues the same order, so a pair with low == high still matches send to receive."""
        d = self.dist
        ops = [d.P2POp(d.isend, send_lo, low, self.group), d.P2POp(d.irecv, recv_hi, high, self.group),
               d.P2POp(d.isend, send_hi, high, self.group), d.P2POp(d.irecv, recv_lo, low, self.group)]
        for w in d.batch_isend_irecv(ops):
            w.wait()

    def sum_(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)

    def max_(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)


# ---- device solvers of the blocks ----------------------------------------------------------

class _DevArray:
    """A raw device pointer as a __cuda_array_interface__ object (for torch.as_tensor)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


@dataclass
class Layout:
    N: tuple          # global interior zones per dimension (nd entries)
    dims: tuple       # ranks per dimension (3 entries)
    x0: tuple
    x1: tuple

    @property
    def nd(self):
        return len(self.N)

    def local(self, rank):
        """(coords, offset, n, lo, hi) of a rank's block."""
        c = coords_of(rank, self.dims)
        off, n, lo, hi = [], [], [], []
        for d in range(self.nd):
            o, m = block(self.N[d], self.dims[d], c[d])
            dx = (self.x1[d] - self.x0[d]) / self.N[d]
            off.append(o)
            n.append(m)
            lo.append(self.x0[d] + o * dx)
            hi.append(self.x0[d] + (o + m) * dx)
        return c, tuple(off), tuple(n), tuple(lo), tuple(hi)

    def split(self):
        return [d for d in range(self.nd) if self.dims[d] > 1]

    def check(self):
        """Every block needs at least Ng zones per dimension (its guards come from its
        immediate neighbours only)."""
        for d in range(self.nd):
            if self.N[d] // self.dims[d] < NG:
                raise ValueError(f"blocks of {self.N[d]} zones over {self.dims[d]} ranks are thinner than Ng = {NG}")
        if any(self.dims[d] != 1 for d in range(self.nd, 3)):
            raise ValueError("unused dimensions cannot be split")


def neighbours(layout: Layout, rank: int, d: int) -> tuple:
    """(low, high) neighbour ranks along dimension d (periodic)."""
    c = list(coords_of(rank, layout.dims))
    lo, hi = list(c), list(c)
    lo[d] = (c[d] - 1) % layout.dims[d]
    hi[d] = (c[d] + 1) % layout.dims[d]
    return rank_of(lo, layout.dims), rank_of(hi, layout.dims)


def exchange_numpy(A: np.ndarray, layout: Layout, rank: int, transport) -> None:
    """Fill the guard layers of one rank's host block A (G0, G1, G2, q) as the device path
    does: unsplit dimensions from the block's own periodic images (the c2p scatter), then
    the split ones, in order, from the neighbours through `transport` (CPU tensors)."""
    import torch
    _, _, n, _, _ = layout.local(rank)
    for d in range(layout.nd):
        if layout.dims[d] == 1:
            periodic_fill(A, d, n[d])
    for d in layout.split():
        low, high = neighbours(layout, rank, d)
        send_lo = torch.from_numpy(pack_slab(A, d, 0, n[d]))
        send_hi = torch.from_numpy(pack_slab(A, d, 1, n[d]))
        recv_lo, recv_hi = torch.empty_like(send_hi), torch.empty_like(send_lo)
        transport.exchange(send_lo, send_hi, recv_lo, recv_hi, low, high)
        unpack_slab(A, recv_lo.numpy(), d, 0, n[d])
        unpack_slab(A, recv_hi.numpy(), d, 1, n[d])


def overlapped_exchange_numpy(truth: np.ndarray, layout: Layout, rank: int, transport) -> np.ndarray:
    """The overlapped schedule on one rank's host block, as the device runs it: the block
    starts unknown (NaN), the boundary shell's zones are converted (copied from `truth`, the
    block's interior) with their images along the unsplit dimensions, the split dimensions'
    slabs are exchanged, then the core's zones are converted with their images.  Returns the
    block; it equals the whole-box periodic fill only if the exchange reads nothing but shell
    zones."""
    _, _, n, _, _ = layout.local(rank)
    nd = layout.nd
    n3 = tuple(n) + (1,) * (3 - nd)
    A = np.full_like(truth, np.nan)
    inner = tuple(slice(NG, NG + n3[d]) if d < nd else slice(None) for d in range(3))
    shell = shell_mask(n3, layout.split())
    for region in (shell, ~shell):
        view = A[inner]
        view[region] = truth[inner][region]
        A[inner] = view
        for d in range(nd):
            if layout.dims[d] == 1:
                periodic_fill(A, d, n[d])
        if region is shell:
            for d in layout.split():
                low, high = neighbours(layout, rank, d)
                import torch
                send_lo = torch.from_numpy(pack_slab(A, d, 0, n[d]))
                send_hi = torch.from_numpy(pack_slab(A, d, 1, n[d]))
                recv_lo, recv_hi = torch.empty_like(send_hi), torch.empty_like(send_lo)
                transport.exchange(send_lo, send_hi, recv_lo, recv_hi, low, high)
                unpack_slab(A, recv_lo.numpy(), d, 0, n[d])
                unpack_slab(A, recv_hi.numpy(), d, 1, n[d])
    return A


class _Block:
    """One rank's solver plus its slab buffers."""

    def __init__(self, scheme, layout: Layout, rank: int, stream):
        import torch
        from .mara import Solver
        self.rank = rank
        self.coords, self.off, self.n, lo, hi = layout.local(rank)
        self.solver = Solver(scheme, self.n, lo, hi, stream=stream)
        lib, h = self.solver.lib, self.solver.h
        self.lib, self.h = lib, h
        ext = (ctypes.c_int * 3)(*[1 if (d < layout.nd and layout.dims[d] > 1) else 0 for d in range(3)])
        tabs = [multiplicity_table(layout.N[d], layout.dims[d], self.coords[d]) for d in layout.split()]
        mult = np.ascontiguousarray(np.concatenate(tabs) if tabs else np.zeros(1, np.int32), dtype=np.int32)
        self.solver._check(lib.mgpu_set_external_guards(h, ext, mult.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        # slab buffers per split dimension: [which][side] send and receive
        self.bufs = {}
        for d in layout.split():
            for which in (0, 1):
                nb = ctypes.c_longlong()
                self.solver._check(lib.mgpu_halo_bytes(h, which, d, ctypes.byref(nb)))
                mk = lambda: torch.empty(nb.value, dtype=torch.uint8, device="cuda")   # noqa: E731
                self.bufs[(d, which)] = {"send": [mk(), mk()], "recv": [mk(), mk()]}
        ep, mp = ctypes.c_void_p(), ctypes.c_void_p()
        self.solver._check(lib.mgpu_reduction_targets(h, ctypes.byref(ep), ctypes.byref(mp)))
        self.errs = torch.as_tensor(_DevArray(ep.value, (5,), "<i4"), device="cuda")
        self.maxl = torch.as_tensor(_DevArray(mp.value, (1,), "<i8"), device="cuda")

    def phase(self, phase, stage=0, dt_mode=0, dt=0.0, cfl=0.0):
        self.solver._check(self.lib.mgpu_advance_phase(self.h, phase, stage, dt_mode, float(dt), float(cfl)))

    def pack(self, which, d, stream=None):
        """The send slabs of dimension d, on the solver's stream or on `stream`."""
        b = self.bufs[(d, which)]
        for side in (0, 1):
            buf = ctypes.c_void_p(b["send"][side].data_ptr())
            if stream is None:
                self.solver._check(self.lib.mgpu_halo_pack(self.h, which, d, side, buf))
            else:
                self.solver._check(self.lib.mgpu_halo_pack_on(self.h, which, d, side, buf,
                                                              ctypes.c_void_p(stream.cuda_stream)))

    def unpack(self, which, d, stream=None):
        b = self.bufs[(d, which)]
        for side in (0, 1):
            buf = ctypes.c_void_p(b["recv"][side].data_ptr())
            if stream is None:
                self.solver._check(self.lib.mgpu_halo_unpack(self.h, which, d, side, buf))
            else:
                self.solver._check(self.lib.mgpu_halo_unpack_on(self.h, which, d, side, buf,
                                                                ctypes.c_void_p(stream.cuda_stream)))


class DecomposedSolver:
    """The blocks of `layout` held by this process (`ranks`), advanced together.

    With a TorchTransport a process holds one rank (ranks = [dist rank]); with transport
    None every rank of the layout lives in this process on the current device (one shared
    stream, slabs copied directly)."""

    def __init__(self, scheme, layout: Layout, ranks, transport=None, stream=None, overlap=True):
        import torch
        layout.check()
        self.layout = layout
        self.scheme = scheme
        self.transport = transport
        self.stream = stream or torch.cuda.Stream()
        # overlap: each stage converts the blocks' boundary shells first (phase 4), exchanges
        # their slabs on a side stream while the cores convert (phase 5), and starts the sweeps
        # once both are done; otherwise c2p, exchange and sweeps run one after the other
        self.overlap = overlap
        self.side = torch.cuda.Stream() if overlap else None
        self.blocks = [_Block(scheme, layout, r, self.stream.cuda_stream) for r in ranks]
        self.by_rank = {b.rank: b for b in self.blocks}
        self.ns = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}[scheme.advance]

    # -- guard exchange of every split dimension, in order x, y, z (on `stream`, or on the
    # solvers' stream) --
    def exchange(self, which, stream=None):
        L = self.layout
        for d in L.split():
            for b in self.blocks:
                b.pack(which, d, stream)
            for b in self.blocks:
                low, high = neighbours(L, b.rank, d)
                buf = b.bufs[(d, which)]
                if self.transport is None:
                    # low neighbour's high slab -> my low guards; high neighbour's low slab -> my high guards
                    buf["recv"][0].copy_(self.by_rank[low].bufs[(d, which)]["send"][1])
                    buf["recv"][1].copy_(self.by_rank[high].bufs[(d, which)]["send"][0])
                else:
                    self.transport.exchange(buf["send"][0], buf["send"][1], buf["recv"][0], buf["recv"][1], low, high)
            for b in self.blocks:
                b.unpack(which, d, stream)

    def _reduce(self):
        import torch
        if self.transport is None:
            errs = torch.stack([b.errs for b in self.blocks]).sum(0)
            maxl = torch.stack([b.maxl for b in self.blocks]).max(0).values
            for b in self.blocks:
                b.errs.copy_(errs)
                b.maxl.copy_(maxl)
        else:
            for b in self.blocks:
                self.transport.sum_(b.errs)
                self.transport.max_(b.maxl)

    def advance(self, dt=None, cfl=None):
        """Enqueue one advance of every block: fixed dt, or (cfl) the global CFL step from the
        previous advance's MaxLambda (maximum over ranks, as get_timestep's MPI minimum of dt).
        Asynchronous; `errors()` reads the outcome."""
        import torch
        dt_mode = 0 if cfl is None else 1
        with torch.cuda.stream(self.stream):
            for b in self.blocks:
                b.phase(0, 0, dt_mode, dt or 0.0, cfl or 0.0)
            for s in range(self.ns):
                if self.overlap:
                    for b in self.blocks:
                        b.phase(4, s)                      # the shells the slabs read
                    self.side.wait_stream(self.stream)
                    with torch.cuda.stream(self.side):
                        self.exchange(0, self.side)         # slabs travel ...
                    for b in self.blocks:
                        b.phase(5, s)                      # ... while the cores convert
                    self.stream.wait_stream(self.side)
                else:
                    for b in self.blocks:
                        b.phase(1, s)
                    self.exchange(0)
                for b in self.blocks:
                    b.phase(2, s)
            for b in self.blocks:
                b.phase(1, self.ns)
            self._reduce()
            for b in self.blocks:
                b.phase(3, 0)

    def synchronize(self):
        self.stream.synchronize()

    def errors(self) -> int:
        """Failed zones of the last advance, summed over ranks (the first failing stage)."""
        self.synchronize()
        e = self.blocks[0].errs.cpu().numpy()
        nz = e[np.nonzero(e)[0]]
        return int(nz[0]) if len(nz) else 0

    def get_timestep(self, cfl: float) -> float:
        self.synchronize()
        return self.blocks[0].solver.get_timestep(cfl)

    def upload_global(self, P: np.ndarray):
        """Scatter a global guarded primitive array (the single-box layout) to the blocks."""
        for b in self.blocks:
            b.solver.upload(np.ascontiguousarray(self._window(P, b)))

    def _window(self, P, b):
        nd = self.layout.nd
        sl = []
        for d in range(3):
            if d < nd:
                sl.append(slice(b.off[d], b.off[d] + b.n[d] + 2 * NG))
            else:
                sl.append(slice(None))
        # the global array with its own periodic guards: block windows include guard layers
        Pg = P.reshape(tuple(v + 2 * NG for v in self.layout.N) + (1,) * (3 - nd) + (8,))
        return Pg[tuple(sl)]

    def download_global(self) -> np.ndarray:
        """Gather the interiors (this process's blocks) into a global guarded array with
        periodic guards."""
        nd = self.layout.nd
        shape = tuple(v + 2 * NG for v in self.layout.N) + (1,) * (3 - nd) + (8,)
        out = np.zeros(shape)
        for b in self.blocks:
            loc = b.solver.download()
            src, dst = [], []
            for d in range(3):
                if d < nd:
                    src.append(slice(NG, NG + b.n[d]))
                    dst.append(slice(NG + b.off[d], NG + b.off[d] + b.n[d]))
                else:
                    src.append(slice(None))
                    dst.append(slice(None))
            out[tuple(dst)] = loc[tuple(src)]
        for d in range(nd):
            periodic_fill(out.reshape(out.shape[:3] + (8,)), d, self.layout.N[d])
        return out

    def close(self):
        for b in self.blocks:
            b.solver.close()
