"""Ensembles of independent boxes of uneven size advanced together on one GPU.

The reference advances one domain per process (its solver is a global singleton,
Mara/mara.cpp:135); a parameter study runs it once per box.  `Ensemble` holds many boxes
with one scheme and advances all of them with one CUDA graph per call: every phase of the
step is one persistent launch walking the tiles of all boxes (ctf_b200/csrc/rmhd_ensemble.cuh),
and box b evolves exactly as a `mara.Solver` of that box would (same kernels' arithmetic,
its own dt, MaxLambda, error count and commit).

The launch shape (tile lengths, CTAs per SM of each launch) is chosen by the library's
autotuner (`mgpu_ensemble_autotune`); `tuned()` keeps the result in a JSON cache keyed by
the device, the scheme and the box sizes, so a set-up is tuned once.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np

from . import _lib
from .mara import MaraError, Scheme, Solver, _dp

CACHE_ENV = "CTF_B200_TUNING_CACHE"


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Ensemble:
    """Boxes `sizes[b]` (tuples of nd ints) on extents x0[b]..x1[b] (default: unit boxes)."""

    def __init__(self, scheme: Scheme, sizes, x0=None, x1=None):
        self.lib = _lib.load()
        self.scheme = scheme
        sizes = [tuple(int(v) for v in s) for s in sizes]
        nd = len(sizes[0])
        if any(len(s) != nd for s in sizes):
            raise MaraError("[Mara] every box of an ensemble has the same dimensionality")
        self.sizes, self.nd, self.nb = sizes, nd, len(sizes)
        N = np.ascontiguousarray(np.array(sizes, dtype=np.int32).reshape(-1))
        lo = None if x0 is None else np.ascontiguousarray(np.asarray(x0, dtype=np.float64).reshape(-1))
        hi = None if x1 is None else np.ascontiguousarray(np.asarray(x1, dtype=np.float64).reshape(-1))
        cfg = scheme.to_config()
        h = ctypes.c_void_p()
        rc = self.lib.mgpu_ensemble_create(ctypes.byref(cfg), nd, self.nb, _ip(N),
                                           None if lo is None else _dp(lo), None if hi is None else _dp(hi),
                                           ctypes.byref(h))
        if rc:
            raise MaraError(f"mgpu_ensemble_create failed ({rc})")
        self.h = h
        self._keep = (N, lo, hi)

    def _check(self, rc):
        if rc:
            raise MaraError(f"[Mara] {self.lib.mgpu_ensemble_last_error(self.h).decode()} (code {rc})")

    def set_stream(self, stream: int):
        """Run on an existing CUDA stream (a cudaStream_t as an int, e.g. torch's
        `Stream.cuda_stream`); the default is the ensemble's own stream."""
        self._check(self.lib.mgpu_ensemble_set_stream(self.h, ctypes.c_void_p(stream)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mgpu_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, b: int):
        n = self.sizes[b]
        return tuple(v + 6 for v in n) + (1,) * (3 - self.nd) + (8,)

    @property
    def total_interior(self) -> int:
        n = ctypes.c_longlong()
        self._check(self.lib.mgpu_ensemble_total_interior(self.h, ctypes.byref(n)))
        return n.value

    def upload(self, b: int, P: np.ndarray):
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.size != int(np.prod(self.shape(b))):
            raise MaraError("[Mara] primitive has the wrong size for the box")
        self._check(self.lib.mgpu_ensemble_upload_prim(self.h, b, _dp(P)))

    def download(self, b: int) -> np.ndarray:
        out = np.empty(self.shape(b))
        self._check(self.lib.mgpu_ensemble_download_prim(self.h, b, _dp(out)))
        return out

    def advance(self, dt=None, nsteps: int = 1, cfl: float | None = None, graph: bool = True):
        """Enqueue nsteps advances: with per-box `dt` (scalar or nb values), or with each box's
        own CFL step (`cfl`, from its previous advance's MaxLambda).  Asynchronous."""
        if (dt is None) == (cfl is None):
            raise MaraError("[Mara] give either dt or cfl")
        if dt is not None:
            d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.nb,)))
            self._check(self.lib.mgpu_ensemble_advance(self.h, nsteps, 0, _dp(d), 0.0, int(graph)))
        else:
            self._check(self.lib.mgpu_ensemble_advance(self.h, nsteps, 1, None, float(cfl), int(graph)))

    def synchronize(self):
        self._check(self.lib.mgpu_ensemble_synchronize(self.h))

    def errors(self) -> np.ndarray:
        out = np.zeros(self.nb, dtype=np.int32)
        self._check(self.lib.mgpu_ensemble_errors(self.h, _ip(out)))
        return out

    def stats(self, b: int) -> dict:
        s = _lib.MgpuStats()
        self._check(self.lib.mgpu_ensemble_get_stats(self.h, b, ctypes.byref(s)))
        return s.as_dict()

    def timesteps(self, cfl: float) -> np.ndarray:
        out = np.zeros(self.nb)
        self._check(self.lib.mgpu_ensemble_get_timesteps(self.h, float(cfl), _dp(out)))
        return out

    # ---- kernel timing (direct advances only) ---------------------------------------------
    def profile_enable(self, capacity: int = 4096):
        self._check(self.lib.mgpu_ensemble_profile_enable(self.h, capacity))

    def profile_disable(self):
        self._check(self.lib.mgpu_ensemble_profile_disable(self.h))

    def profile_read(self) -> dict:
        """Per kernel class: summed ms, launches and work units since the last read."""
        ms = (ctypes.c_double * 6)()
        ln = (ctypes.c_longlong * 6)()
        un = (ctypes.c_longlong * 6)()
        self._check(self.lib.mgpu_ensemble_profile_read(self.h, ms, ln, un))
        return {k: {"ms": ms[i], "launches": ln[i], "units": un[i]}
                for i, k in enumerate(Solver.KERNEL_CLASSES)}

    # ---- launch shape ------------------------------------------------------------------
    @property
    def launch(self) -> dict:
        L = _lib.MgpuEnsembleLaunch()
        self._check(self.lib.mgpu_ensemble_get_launch(self.h, ctypes.byref(L)))
        return L.as_dict()

    @launch.setter
    def launch(self, shape: dict):
        L = _lib.MgpuEnsembleLaunch(**shape)
        self._check(self.lib.mgpu_ensemble_set_launch(self.h, ctypes.byref(L)))

    def time_advance(self, dt, shape: dict | None = None, reps: int = 5) -> float:
        """Mean device ms of one advance with launch shape `shape`; commits nothing."""
        L = _lib.MgpuEnsembleLaunch(**(shape or self.launch))
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.nb,)))
        ms = ctypes.c_double()
        self._check(self.lib.mgpu_ensemble_time_advance(self.h, ctypes.byref(L), _dp(d), reps, ctypes.byref(ms)))
        return ms.value

    def autotune(self, dt, reps: int = 3) -> tuple[dict, float]:
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.nb,)))
        L = _lib.MgpuEnsembleLaunch()
        ms = ctypes.c_double()
        self._check(self.lib.mgpu_ensemble_autotune(self.h, _dp(d), reps, ctypes.byref(L), ctypes.byref(ms)))
        return L.as_dict(), ms.value

    def tuning_key(self) -> str:
        import torch
        dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
        s = self.scheme
        sig = json.dumps([dev, s.precision, s.extrap, s.riemann, s.advance, self.nd, sorted(self.sizes)])
        return hashlib.sha1(sig.encode()).hexdigest()

    def tuned(self, dt, reps: int = 3, cache: str | None = None) -> dict:
        """Install the cached launch shape for this set-up, or autotune and cache it."""
        path = cache or os.environ.get(CACHE_ENV) or os.path.join(
            os.path.expanduser("~"), ".cache", "ctf_b200", "ensemble_tuning.json")
        key = self.tuning_key()
        db = {}
        if os.path.exists(path):
            try:
                with open(path) as f:
                    db = json.load(f)
            except (OSError, ValueError):
                db = {}
        if key in db:
            self.launch = db[key]["launch"]
            return db[key]
        shape, ms = self.autotune(dt, reps)
        db[key] = {"launch": shape, "ms": ms}
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1)
        os.replace(tmp, path)
        return db[key]


def kh_sizes(nboxes: int = 256, seed: int = 0, lo: int = 64, hi: int = 512, multiple: int = 8):
    """Box sizes log-uniform in lo^2..hi^2 (square boxes, sides rounded to a multiple of 8)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(lo), np.log(hi), nboxes))
    sides = np.clip(np.round(sides / multiple) * multiple, multiple, None).astype(int)
    return [(int(n), int(n)) for n in sides]
