"""Train the learned c2p initial guess on states the FP64 method produces (run on a GPU).

    python -m ctf_b200.train_c2p [--out ctf_b200/data/c2p_net.npz] [--samples 12000000]

Data: the (conserved, primitive) pairs of FP64 runs of the two turbulence set-ups --
the 64^3 box with PLM + HLLD + RK2 (20 steps, harvested every 5) and the 256^3 box with
WENO5 + HLLD + RK3 (harvested after steps 1, 3 and 5) -- subsampled without replacement to
`--samples` pairs.  Training: minibatch Adam on the device (`mgpu_mlp_train`), learning rate
decaying geometrically.  The result (packed float32 parameters plus provenance) is written
to `--out`; `load()` reads it back.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "c2p_net.npz")


def load(path: str = DEFAULT_OUT) -> np.ndarray:
    """Packed float32 parameters of the trained network."""
    return np.load(path)["params"].astype(np.float32)


def harvest_runs(seed=0):
    import torch
    from . import ics, learned_c2p as lc
    from .mara import Scheme, Solver
    Xs, Ys, runs = [], [], []
    plan = [((64, 64, 64), dict(extrap="plm", riemann="hlld", advance="rk2"), 20, {5, 10, 15, 20}),
            ((256, 256, 256), dict(extrap="weno5", riemann="hlld", advance="rk3"), 5, {1, 3, 5})]
    for n, kw, steps, at in plan:
        s = Solver(Scheme(**kw), n)
        s.upload(ics.turbulence_box(n, seed=seed))
        assert s.advance(0.0) == 0
        for k in range(1, steps + 1):
            e = s.advance(s.get_timestep(0.3))
            if e:
                raise RuntimeError(f"FP64 run failed at step {k}: {e} zones")
            if k in at:
                X, Y = lc.harvest(s)
                Xs.append(X)
                Ys.append(Y)
        runs.append(f"{n[0]}^3 {kw} steps {sorted(at)}")
        s.close()
        torch.cuda.synchronize()
    return torch.cat(Xs), torch.cat(Ys), runs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--samples", type=int, default=12_000_000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import torch
    from . import learned_c2p as lc
    torch.cuda.set_device(0)
    t0 = time.time()
    X, Y, runs = harvest_runs(args.seed)
    n_all = X.shape[0]
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    if n_all > args.samples:
        idx = torch.randperm(n_all, device="cuda", generator=g)[: args.samples]
        X, Y = X[idx].contiguous(), Y[idx].contiguous()
    t1 = time.time()
    params, losses = lc.train(X, Y, steps=args.steps, batch=args.batch, seed=args.seed)
    t2 = time.time()
    final_loss, _ = lc.loss_grad(params, X[:1_000_000], Y[:1_000_000])
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez(args.out, params=params, losses=np.array(losses), samples=X.shape[0], harvested=n_all,
             runs=np.array(runs), final_loss=final_loss, train_seconds=t2 - t1, harvest_seconds=t1 - t0)
    print(f"harvested {n_all} pairs ({t1 - t0:.1f} s), trained on {X.shape[0]} for {args.steps} steps "
          f"({t2 - t1:.1f} s); loss {losses[0]:.3e} -> {losses[-1]:.3e}; full-data loss {final_loss:.3e}")


if __name__ == "__main__":
    main()
