"""FP64 numpy oracle of the learned c2p network (test infrastructure only).

The network maps five scale-free features of the c2p invariants (D, tau, S^2, B^2,
(S.B)^2) to (log W, log h), from which the Newton polish starts at W and Z = D W h.
It has no counterpart in the reference; it restates the forward pass, the MSE loss, its
gradient and one Adam update exactly as the CUDA kernels in ctf_b200/csrc/c2p_mlp.cu do,
so that their gradients can be checked.

Packed parameter layout (float32 on the device, float64 here), in order:
  W1[64,5] b1[64] W2[64,64] b2[64] W3[64,64] b3[64] W4[2,64] b4[2]
  xmean[5] xstd[5] ymean[2] ystd[2]
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 5, 64, 2
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)),
          ("b3", (NH,)), ("W4", (NOUT, NH)), ("b4", (NOUT,)), ("xmean", (NIN,)), ("xstd", (NIN,)),
          ("ymean", (NOUT,)), ("ystd", (NOUT,))]
N_TRAIN = sum(int(np.prod(s)) for n, s in SHAPES[:8])          # 8834 trainable
N_PARAMS = sum(int(np.prod(s)) for n, s in SHAPES)             # 8848 with normalisation


def unpack(p):
    out, o = {}, 0
    for n, s in SHAPES:
        k = int(np.prod(s))
        out[n] = np.asarray(p[o:o + k], dtype=np.float64).reshape(s)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[n], dtype=np.float64).ravel() for n, _ in SHAPES])


def init_params(rng, xmean, xstd, ymean, ystd):
    d = {}
    for n, s in SHAPES[:8]:
        if n.startswith("W"):
            d[n] = rng.standard_normal(s) * np.sqrt(1.0 / s[1])
        else:
            d[n] = np.zeros(s)
    d["xmean"], d["xstd"], d["ymean"], d["ystd"] = xmean, xstd, ymean, ystd
    return pack(d)


def features(U, gamma=4.0 / 3.0):
    """Scale-free features of the c2p invariants from conserved states U[n, 8]."""
    D, tau = U[:, 0], U[:, 1]
    S = U[:, 2:5]
    B = U[:, 5:8]
    S2 = np.sum(S * S, axis=1)
    B2 = np.sum(B * B, axis=1)
    SB = np.sum(S * B, axis=1)
    SB2 = SB * SB
    return np.stack([np.log1p(tau / D), np.log1p(S2 / (D * D)), np.log1p(B2 / D),
                     np.log1p(SB2 / (D * D * D)), SB2 / (S2 * B2 + 1e-30)], axis=1)


def targets(P, gamma=4.0 / 3.0):
    """(log W, log h) of primitive states P[n, 8]."""
    v2 = np.sum(P[:, 2:5] ** 2, axis=1)
    W = 1.0 / np.sqrt(1.0 - v2)
    h = 1.0 + gamma / (gamma - 1.0) * P[:, 1] / P[:, 0]
    return np.stack([np.log(W), np.log(h)], axis=1)


def forward(p, X):
    d = unpack(p)
    x = (X - d["xmean"]) / d["xstd"]
    a1 = np.tanh(x @ d["W1"].T + d["b1"])
    a2 = np.tanh(a1 @ d["W2"].T + d["b2"])
    a3 = np.tanh(a2 @ d["W3"].T + d["b3"])
    yn = a3 @ d["W4"].T + d["b4"]
    return yn * d["ystd"] + d["ymean"], (x, a1, a2, a3, yn)


def loss_grad(p, X, Y):
    """Mean squared error over the normalised outputs and its gradient w.r.t. the 8834
    trainable parameters (normalisation constants are fixed)."""
    d = unpack(p)
    _, (x, a1, a2, a3, yn) = forward(p, X)
    tn = (Y - d["ymean"]) / d["ystd"]
    n = X.shape[0]
    r = yn - tn
    loss = np.sum(r * r) / (n * NOUT)
    g_yn = 2.0 * r / (n * NOUT)
    gW4 = g_yn.T @ a3
    gb4 = g_yn.sum(0)
    g3 = (g_yn @ d["W4"]) * (1 - a3 * a3)
    gW3 = g3.T @ a2
    gb3 = g3.sum(0)
    g2 = (g3 @ d["W3"]) * (1 - a2 * a2)
    gW2 = g2.T @ a1
    gb2 = g2.sum(0)
    g1 = (g2 @ d["W2"]) * (1 - a1 * a1)
    gW1 = g1.T @ x
    gb1 = g1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3, gW4.ravel(), gb4])
    return loss, grad


def adam_step(p, grad, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trainable prefix of p (t counts from 1)."""
    p = p.copy()
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    p[:N_TRAIN] -= lr * mh / (np.sqrt(vh) + eps)
    return p, m, v
