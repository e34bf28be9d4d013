"""Checkpoints of the primitive state, in the layout of the reference's Lua drivers.

The reference writes `data/<run>/chkpt.<NNNN>.h5` with a group `prim` holding one dataset per
primitive name (rho, pre, vx, vy, vz, Bx, By, Bz) over the global interior, and the string
datasets `status`, `measure_log`, `git_sha` and `model_parameters` as JSON
(ctf-core/run-mara.lua:179-204, ctf-core/drvtrb.lua:510-582).  HDF5 is not available in
this image, so the same content is written as a directory:

    <path>/prim/<name>.bin      float64, C order, the global interior shape
    <path>/checkpoint.json      {"shape", "prim_names", "status", "measure_log",
                                 "git_sha", "model_parameters"}

`write` takes a guarded AoS primitive array (the layout `Mara.advance` uses); `read` returns
one with the periodic guard layers filled, ready for `Solver.upload`.  With h5py installed,
`write_h5`/`read_h5` use the reference's HDF5 layout itself.
"""
from __future__ import annotations

import json
import os

import numpy as np

PRIM_NAMES = ("rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz")   # Rmhd::GetPrimNames
NG = 3


def with_periodic_guards(I: np.ndarray, nd: int) -> np.ndarray:
    """Interior (n..., 8) -> guarded (G0, G1, G2, 8) with periodic guards, unused dimensions
    of extent 1 (the Solver layout)."""
    pad = [(NG, NG)] * nd + [(0, 0)]
    P = np.pad(I, pad, mode="wrap")
    return np.ascontiguousarray(P.reshape(P.shape[:nd] + (1,) * (3 - nd) + (8,)))


def _split(P: np.ndarray, nd: int):
    """Guarded AoS (G0[, G1[, G2]], [1,] 8) -> interior (n..., 8)."""
    Q = P.reshape(P.shape[:nd] + (-1,)) if P.ndim > nd + 1 else P
    Q = Q.reshape(Q.shape[:nd] + (8,))
    return Q[tuple(slice(NG, -NG) for _ in range(nd))]


def write(path: str, P: np.ndarray, nd: int, status: dict | None = None, measure_log=None,
          model_parameters: dict | None = None, git_sha: str = "b200") -> None:
    I = np.ascontiguousarray(_split(np.asarray(P, dtype=np.float64), nd))
    os.makedirs(os.path.join(path, "prim"), exist_ok=True)
    for q, name in enumerate(PRIM_NAMES):
        np.ascontiguousarray(I[..., q]).tofile(os.path.join(path, "prim", name + ".bin"))
    meta = {"shape": list(I.shape[:nd]), "prim_names": list(PRIM_NAMES), "status": status or {},
            "measure_log": measure_log or [], "git_sha": git_sha, "model_parameters": model_parameters}
    tmp = os.path.join(path, "checkpoint.json.tmp")
    with open(tmp, "w") as f:
        json.dump(meta, f, indent=1)
    os.replace(tmp, os.path.join(path, "checkpoint.json"))


def read(path: str):
    """-> (guarded AoS primitives with periodic guards, metadata dict)."""
    with open(os.path.join(path, "checkpoint.json")) as f:
        meta = json.load(f)
    shape = tuple(meta["shape"])
    nd = len(shape)
    I = np.empty(shape + (8,))
    for q, name in enumerate(meta["prim_names"]):
        I[..., q] = np.fromfile(os.path.join(path, "prim", name + ".bin"), dtype=np.float64).reshape(shape)
    return with_periodic_guards(I, nd), meta


def write_h5(fname: str, P: np.ndarray, nd: int, status: dict | None = None, measure_log=None,
             model_parameters: dict | None = None, git_sha: str = "b200") -> None:
    import h5py   # not in this image; the reference's own layout when available
    I = _split(np.asarray(P, dtype=np.float64), nd)
    with h5py.File(fname, "w") as f:
        g = f.create_group("prim")
        for q, name in enumerate(PRIM_NAMES):
            g[name] = I[..., q]
        f["status"] = json.dumps(status or {})
        f["measure_log"] = json.dumps(measure_log or [])
        f["git_sha"] = git_sha
        if model_parameters:
            f["model_parameters"] = json.dumps(model_parameters)


def read_h5(fname: str):
    import h5py
    with h5py.File(fname, "r") as f:
        I = np.stack([f["prim"][name][...] for name in PRIM_NAMES], axis=-1)
        meta = {k: json.loads(f[k][()]) for k in ("status", "measure_log") if k in f}
    return with_periodic_guards(I, I.ndim - 1), meta
