"""Learned c2p initial guess: harvest, training and installation (no reference counterpart).

The network (``ctf_b200/csrc/c2p_mlp_net.cuh``) maps five scale-free features of the c2p
invariants (D, tau, S^2, B^2, (S.B)^2) to (log W, log h).  It is trained on the
(conserved, primitive) pairs that the method itself produces: :func:`harvest` reads them
off a solver's committed state after FP64 runs.  Training runs on the device with the
library's own forward/backward/Adam kernels (``mgpu_mlp_train``); torch only provides the
device buffers.  Installed with ``Solver.set_c2p_network`` and enabled by
``Scheme(learned_c2p=True)``, the network seeds the first Newton attempt of every c2p; the
FP64 Newton polish decides the result and the reference's four-attempt ladder runs whenever
that attempt fails.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

NIN, NH, NOUT = 5, 64, 2
N_TRAIN = NH * NIN + NH + NH * NH + NH + NH * NH + NH + NOUT * NH + NOUT


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def n_params() -> int:
    return _lib.load().mgpu_mlp_param_count()


def harvest(solver):
    """Features (n x 5) and targets (n x 2) of every interior zone of the solver's state,
    as float32 torch tensors on the current device."""
    import torch
    lib = _lib.load()
    n = int(np.prod(solver.n))
    X = torch.empty((n, NIN), dtype=torch.float32, device="cuda")
    Y = torch.empty((n, NOUT), dtype=torch.float32, device="cuda")
    cnt = ctypes.c_longlong()
    solver._check(lib.mgpu_c2p_harvest(solver.h, _ptr(X), _ptr(Y), n, ctypes.byref(cnt)))
    return X, Y


def init_params(X, Y, seed: int = 0) -> np.ndarray:
    """Random weights (scaled by fan-in) and the standardisation constants of the data."""
    rng = np.random.default_rng(seed)
    Xh = X.double().cpu().numpy()
    Yh = Y.double().cpu().numpy()
    parts = []
    for shape in [(NH, NIN), (NH,), (NH, NH), (NH,), (NH, NH), (NH,), (NOUT, NH), (NOUT,)]:
        if len(shape) == 2:
            parts.append(rng.standard_normal(shape).ravel() * np.sqrt(1.0 / shape[1]))
        else:
            parts.append(np.zeros(shape))
    xs = Xh.std(0)
    ys = Yh.std(0)
    parts += [Xh.mean(0), np.where(xs > 0, xs, 1.0), Yh.mean(0), np.where(ys > 0, ys, 1.0)]
    return np.concatenate(parts).astype(np.float32)


def train(X, Y, params: np.ndarray | None = None, steps: int = 2000, batch: int = 16384,
          lr: float = 2e-3, lr_final: float = 1e-4, seed: int = 0, chunk: int = 100):
    """Minibatch Adam on the device; returns (params as float32 numpy, loss history)."""
    import torch
    lib = _lib.load()
    n = X.shape[0]
    p0 = init_params(X, Y, seed) if params is None else np.asarray(params, np.float32)
    P = torch.tensor(p0, device="cuda")
    M = torch.zeros(N_TRAIN, dtype=torch.float32, device="cuda")
    V = torch.zeros(N_TRAIN, dtype=torch.float32, device="cuda")
    work = torch.empty(int(lib.mgpu_mlp_work_floats(batch)), dtype=torch.float32, device="cuda")
    losses = []
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        frac = done / max(steps - 1, 1)
        lr_k = lr * (lr_final / lr) ** frac        # geometric decay
        loss = ctypes.c_double()
        rc = lib.mgpu_mlp_train(_ptr(P), _ptr(M), _ptr(V), _ptr(X), _ptr(Y), n, batch, k,
                                ctypes.c_float(lr_k), done, _ptr(work), ctypes.byref(loss))
        if rc:
            raise RuntimeError(f"mgpu_mlp_train failed ({rc})")
        losses.append(loss.value)
        done += k
    return P.cpu().numpy(), losses


def loss_grad(params, X, Y):
    """Loss and gradient over all of (X, Y) with the device kernels (for checks)."""
    import torch
    lib = _lib.load()
    n = X.shape[0]
    P = torch.tensor(np.asarray(params, np.float32), device="cuda")
    G = torch.empty(N_TRAIN, dtype=torch.float32, device="cuda")
    work = torch.empty(int(lib.mgpu_mlp_work_floats(n)), dtype=torch.float32, device="cuda")
    loss = ctypes.c_double()
    rc = lib.mgpu_mlp_loss_grad(_ptr(P), _ptr(X), _ptr(Y), n, _ptr(G), _ptr(work), ctypes.byref(loss))
    if rc:
        raise RuntimeError(f"mgpu_mlp_loss_grad failed ({rc})")
    return loss.value, G.cpu().numpy()


def forward(params, X):
    import torch
    lib = _lib.load()
    P = torch.tensor(np.asarray(params, np.float32), device="cuda")
    Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device="cuda")
    rc = lib.mgpu_mlp_forward(_ptr(P), _ptr(X), X.shape[0], _ptr(Y))
    if rc:
        raise RuntimeError(f"mgpu_mlp_forward failed ({rc})")
    return Y
