"""The learned c2p initial guess: the device kernels against the FP64 numpy oracle
(oracle/mlp.py), the harvest against the host computation, and what the trained network
gains over the method without it."""
import numpy as np
import pytest

from ctf_b200 import ics, learned_c2p as lc
from ctf_b200.mara import Scheme, Solver
from oracle import PortOracle, Scheme as OScheme
from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def _data(n=4096, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    X = np.stack([rng.uniform(0, 3, n), rng.uniform(0, 4, n), rng.uniform(0, 2, n),
                  rng.uniform(0, 5, n), rng.uniform(0, 1, n)], axis=1)
    Y = np.stack([rng.uniform(0, 2, n), rng.uniform(0, 1.5, n)], axis=1)
    return torch.tensor(X, dtype=torch.float32, device="cuda"), torch.tensor(Y, dtype=torch.float32,
                                                                              device="cuda")


def test_forward_and_gradient_match_fp64_oracle():
    X, Y = _data()
    p = lc.init_params(X, Y, seed=3)
    Xh, Yh = X.double().cpu().numpy(), Y.double().cpu().numpy()
    # forward
    y_dev = lc.forward(p, X).double().cpu().numpy()
    y_ref, _ = omlp.forward(p.astype(np.float64), Xh)
    assert np.abs(y_dev - y_ref).max() <= 1e-4 * max(1.0, np.abs(y_ref).max())
    # loss and gradient (FP32 accumulation on the device vs FP64 here)
    loss, g = lc.loss_grad(p, X, Y)
    loss_ref, g_ref = omlp.loss_grad(p.astype(np.float64), Xh, Yh)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    # directional check of the oracle gradient itself (central difference in FP64)
    rng = np.random.default_rng(1)
    d = rng.standard_normal(omlp.N_TRAIN)
    eps = 1e-6
    pp = p.astype(np.float64).copy()
    pm = pp.copy()
    pp[:omlp.N_TRAIN] += eps * d
    pm[:omlp.N_TRAIN] -= eps * d
    fd = (omlp.loss_grad(pp, Xh, Yh)[0] - omlp.loss_grad(pm, Xh, Yh)[0]) / (2 * eps)
    assert abs(fd - g_ref @ d) <= 1e-6 * max(1.0, abs(fd))


def test_tensor_core_forward_matches_fp32_forward():
    """The tcgen05 path (BF16 weights and activations, FP32 accumulation in TMEM) against the
    per-thread FP32 evaluation of the same network, on 3 tiles of 128 rows plus a ragged one."""
    import ctypes
    import torch
    from ctf_b200 import _lib
    X, Y = _data(n=128 * 3 + 37, seed=9)
    p = lc.init_params(X, Y, seed=10)
    # make the hidden layers matter: larger weights than the fan-in initialisation
    p[:lc.N_TRAIN] *= 2.0
    y32 = lc.forward(p, X).cpu().numpy()
    ytc = torch.empty_like(Y)
    lib = _lib.load()
    rc = lib.mgpu_mlp_forward_tc(p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 ctypes.c_void_p(X.data_ptr()), X.shape[0], ctypes.c_void_p(ytc.data_ptr()))
    assert rc == 0
    ytc = ytc.cpu().numpy()
    assert np.all(np.isfinite(ytc))
    ystd = p[-2:]
    err = np.abs(ytc - y32) / ystd          # in units of the output spread
    assert err.max() <= 0.08 and err.mean() <= 0.02, (err.max(), err.mean())


def test_one_adam_step_matches_oracle():
    X, Y = _data(n=2048, seed=4)
    p0 = lc.init_params(X, Y, seed=5)
    p1, _ = lc.train(X, Y, params=p0, steps=1, batch=2048, lr=1e-3, lr_final=1e-3)
    _, g = omlp.loss_grad(p0.astype(np.float64), X.double().cpu().numpy(), Y.double().cpu().numpy())
    ref, _, _ = omlp.adam_step(p0.astype(np.float64), g, np.zeros_like(g), np.zeros_like(g), 1, 1e-3)
    assert np.abs(p1 - ref).max() <= 1e-5


def test_harvest_matches_host_features():
    n = (12, 10, 8)
    P0 = ics.turbulence_box(n, seed=41)
    s = Solver(Scheme(), n)
    s.upload(P0)
    X, Y = lc.harvest(s)
    P = P0[3:-3, 3:-3, 3:-3].reshape(-1, 8)
    port = PortOracle(OScheme(n=n))
    U = np.array([port.prim_to_cons(p)[0] for p in P])
    assert np.abs(X.cpu().numpy() - omlp.features(U)).max() <= 1e-5
    assert np.abs(Y.cpu().numpy() - omlp.targets(P)).max() <= 1e-6


@pytest.fixture(scope="module")
def trained():
    """Train on states the method produced: 40 FP64 steps of two 32^3 turbulence boxes."""
    import torch
    Xs, Ys = [], []
    for seed, kw in ((50, dict()), (51, dict(extrap="weno5", advance="rk3"))):
        n = (32, 32, 32)
        s = Solver(Scheme(**kw), n)
        s.upload(ics.turbulence_box(n, seed=seed, vrms=0.5))
        assert s.advance(0.0) == 0
        for k in range(20):
            assert s.advance(s.get_timestep(0.3)) == 0
            if k % 5 == 4:
                X, Y = lc.harvest(s)
                Xs.append(X)
                Ys.append(Y)
    X = torch.cat(Xs)
    Y = torch.cat(Ys)
    params, losses = lc.train(X, Y, steps=1500, batch=8192)
    return params, losses


def test_training_reduces_the_loss(trained):
    params, losses = trained
    assert losses[-1] < 0.05 * losses[0], losses


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_learned_guess_gains_over_the_method_without_it(trained, precision):
    """Same step with and without the network: the Newton polish lands on the same state
    (FP64 Newton to 1e-12) and the network cuts the zone c2p's Newton iterations."""
    params, _ = trained
    n = (32, 32, 32)
    P0 = ics.turbulence_box(n, seed=77, vrms=0.5)
    out, its = {}, {}
    for learned in (False, True):
        s = Solver(Scheme(precision=precision, learned_c2p=learned), n)
        s.set_c2p_network(params)
        s.upload(P0.copy())
        assert s.advance(0.0) == 0
        dt = s.get_timestep(0.3)
        assert s.advance(dt) == 0
        st = s.stats()
        its[learned] = st["c2p_iters"] / st["c2p_calls"]
        out[learned] = s.download()
    rel = np.abs(out[True] - out[False]).max() / np.abs(out[False]).max()
    assert rel <= (1e-9 if precision == "fp64" else 1e-5), rel
    assert its[True] < 0.8 * its[False], its


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_learned_guess_under_the_ctu_operator(trained, precision):
    """The learned guess with the CTU-Hancock operator (plm-muscl, the driven-turbulence
    driver's scheme), whose passes write the face array the network's guesses are kept in
    during the c2p: two steps land on the state the plain ladder gives."""
    params, _ = trained
    n = (24, 20, 16)
    P0 = ics.turbulence_box(n, seed=78, vrms=0.3)
    out, its = {}, {}
    for learned in (False, True):
        s = Solver(Scheme(precision=precision, learned_c2p=learned, godunov="plm-muscl", advance="single"), n)
        s.set_c2p_network(params)
        s.upload(P0.copy())
        assert s.advance(0.0) == 0
        dt = s.get_timestep(0.24)
        assert s.advance(dt) == 0 and s.advance(dt) == 0
        st = s.stats()
        its[learned] = st["c2p_iters"] / st["c2p_calls"]
        out[learned] = s.download()
    rel = np.abs(out[True] - out[False]).max() / np.abs(out[False]).max()
    assert rel <= (1e-9 if precision == "fp64" else 1e-5), rel
    assert its[True] < its[False], its
