"""Seeded synthetic initial conditions for the RMHD boxes (host-side IC tooling, numpy).

All states are returned in the reference's AoS primitive layout with guard zones,
``(G0, G1, G2, 8)`` float64, components ``rho, pre, vx, vy, vz, Bx, By, Bz``
(``Mara/rmhd.hpp:20``); the guard zones are filled periodically.

* :func:`turbulence_box` -- rho = 1, p = 1, velocity a Gaussian random field with per-mode
  power ~ |k|^-2 over 1 <= |k| <= 4, rms 0.3, clipped to |v| < 0.9; B = (0, 0, B0) plus a
  perturbation of the same spectrum, rms 0.1, projected so that the corner-centred
  divergence of ``Mara.measure.mean_max_divB`` (``Mara/mara.cpp:2264-2324``) vanishes.
* :func:`stress_box` -- the high-magnetisation set-up: rho = 1, p = 0.01, Lorentz factors
  and magnetisations drawn log-uniform through the CDF of smooth random fields.
* :func:`kh_box` -- 2D relativistic Kelvin-Helmholtz layer (shear layers at y = 1/4, 3/4).
"""
from __future__ import annotations

import numpy as np

NG = 3


def _kgrid(n):
    ks = [np.fft.fftfreq(m, 1.0 / m) for m in n]
    return np.meshgrid(*ks, indexing="ij")


def _random_field(rng, n, kmin, kmax, ncomp, slope=-2.0):
    """Real Gaussian random field on an n-grid, per-mode power ~ |k|^slope on kmin..kmax."""
    K = _kgrid(n)
    kk = np.sqrt(sum(k * k for k in K))
    shell = (kk >= kmin) & (kk <= kmax)
    amp = np.zeros_like(kk)
    amp[shell] = kk[shell] ** (slope / 2.0)
    out = []
    for _ in range(ncomp):
        z = rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)
        out.append(np.fft.ifftn(z * amp).real)
    return np.stack(out, axis=-1), K


def _corner_project(Bhat, K, n):
    """Remove the part of B^(k) seen by the corner divergence stencil of mean_max_divB.

    For cell-centred B the stencil's symbol is d(k)_x = sin(kx dx/2) cos(ky dy/2)
    cos(kz dz/2) (cyclic), up to a common phase; subtracting (d.B^) d / |d|^2 makes the
    discrete divergence vanish to round-off.
    """
    th = [2 * np.pi * K[i] / n[i] for i in range(len(n))]
    s = [np.sin(t / 2) for t in th]
    c = [np.cos(t / 2) for t in th]
    nd = len(n)
    d = []
    for i in range(nd):
        v = s[i].copy()
        for j in range(nd):
            if j != i:
                v = v * c[j]
        d.append(v)
    dd = sum(x * x for x in d)
    dB = sum(d[i] * Bhat[..., i] for i in range(nd))
    safe = np.where(dd > 0, dd, 1.0)
    for i in range(nd):
        Bhat[..., i] = Bhat[..., i] - np.where(dd > 0, d[i] * dB / safe, 0.0)
    return Bhat


def _solenoidal(rng, n, kmin, kmax, rms):
    nd = len(n)
    A, K = _random_field(rng, n, kmin, kmax, nd)
    Bhat = np.stack([np.fft.fftn(A[..., i]) for i in range(nd)], axis=-1)
    Bhat = _corner_project(Bhat, K, n)
    B = np.stack([np.fft.ifftn(Bhat[..., i]).real for i in range(nd)], axis=-1)
    B -= B.mean(axis=tuple(range(nd)))
    B *= rms / np.sqrt(np.mean(np.sum(B * B, axis=-1)))
    return B


def with_guards(interior: np.ndarray, ng: int = NG) -> np.ndarray:
    """Embed an interior prim array (n..., 8) into a periodic guard-zone array."""
    nd = interior.ndim - 1
    pad = [(ng, ng)] * nd + [(0, 0)]
    P = np.pad(interior, pad, mode="wrap")
    if nd < 3:
        P = P.reshape(P.shape[:nd] + (1,) * (3 - nd) + (8,))
    return np.ascontiguousarray(P)


def interior(P: np.ndarray, nd: int = 3, ng: int = NG) -> np.ndarray:
    sl = tuple(slice(ng, -ng) if d < nd else slice(None) for d in range(3))
    return P[sl]


def turbulence_box(n=(64, 64, 64), seed=0, vrms=0.3, vmax=0.9, B0=1.0, dBrms=0.1,
                   rho=1.0, pre=1.0, kmin=1.0, kmax=4.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = tuple(n)
    nd = len(n)
    v, _ = _random_field(rng, n, kmin, kmax, 3)
    v -= v.mean(axis=tuple(range(nd)))
    v *= vrms / np.sqrt(np.mean(np.sum(v * v, axis=-1)))
    speed = np.sqrt(np.sum(v * v, axis=-1))
    over = speed >= vmax
    v[over] *= ((vmax - 1e-6) / speed[over])[:, None]
    B = np.zeros(n + (3,))
    B[..., 2 if nd == 3 else 0] = B0
    if dBrms > 0:
        dB = _solenoidal(rng, n, kmin, kmax, dBrms)
        B[..., :nd] += dB
    P = np.zeros(n + (8,))
    P[..., 0] = rho
    P[..., 1] = pre
    P[..., 2:5] = v
    P[..., 5:8] = B
    return with_guards(P)


def _loguniform_field(rng, n, lo, hi, kmin=1.0, kmax=4.0):
    f, _ = _random_field(rng, n, kmin, kmax, 1)
    f = f[..., 0]
    ranks = np.argsort(np.argsort(f.ravel())).reshape(f.shape)
    u = (ranks + 0.5) / f.size
    return np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))


def stress_box(n=(64, 64, 64), seed=0, gamma=4.0 / 3.0, rho=1.0, pre=0.01,
               W_range=(1.0, 10.0), sigma_range=(0.1, 10.0)) -> np.ndarray:
    """High-magnetisation box: W and sigma = B^2/(rho h) log-uniform over their ranges."""
    rng = np.random.default_rng(seed)
    n = tuple(n)
    W = _loguniform_field(rng, n, *W_range)
    vdir, _ = _random_field(rng, n, 1.0, 4.0, 3)
    vdir /= np.sqrt(np.sum(vdir * vdir, axis=-1, keepdims=True)) + 1e-300
    vmag = np.sqrt(1.0 - 1.0 / (W * W))
    v = vdir * vmag[..., None]
    h = 1.0 + gamma / (gamma - 1.0) * pre / rho
    sigma = _loguniform_field(rng, n, *sigma_range)
    Bmag = np.sqrt(sigma * rho * h)
    B = _solenoidal(rng, n, 1.0, 4.0, 1.0)
    B *= (Bmag / (np.sqrt(np.sum(B * B, axis=-1)) + 1e-300))[..., None]
    # rescaling per zone breaks the discrete constraint: project once more
    nd = len(n)
    K = _kgrid(n)
    Bhat = np.stack([np.fft.fftn(B[..., i]) for i in range(nd)], axis=-1)
    Bhat = _corner_project(Bhat, K, n)
    B = np.stack([np.fft.ifftn(Bhat[..., i]).real for i in range(nd)], axis=-1)
    P = np.zeros(n + (8,))
    P[..., 0] = rho
    P[..., 1] = pre
    P[..., 2:5] = v
    P[..., 5:8] = B
    return with_guards(P)


def kh_box(n=(64, 64), seed=0, shear=0.25, width=0.01, rho=(1.0, 2.0), pre=1.0,
           Bx=0.01, amp=1e-2) -> np.ndarray:
    """2D RMHD Kelvin-Helmholtz layer on the unit square (layers at y = 1/4 and 3/4)."""
    rng = np.random.default_rng(seed)
    nx, ny = n
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    prof = np.tanh((Y - 0.25) / width) - np.tanh((Y - 0.75) / width) - 1.0
    P = np.zeros((nx, ny, 8))
    P[..., 0] = rho[0] + (rho[1] - rho[0]) * 0.5 * (1.0 - prof)
    P[..., 1] = pre
    P[..., 2] = shear * prof
    phases = rng.uniform(0, 2 * np.pi, size=4)
    pert = sum(np.sin(2 * np.pi * (m + 1) * X + phases[m]) for m in range(4)) / 4.0
    env = np.exp(-((Y - 0.25) / 0.05) ** 2) + np.exp(-((Y - 0.75) / 0.05) ** 2)
    P[..., 3] = amp * pert * env
    P[..., 5] = Bx
    return with_guards(P)
