"""FP32-bulk (optionally + learned c2p) against the plain FP64 path over many steps.

    python -m ctf_b200.accuracy [--n 512] [--steps 100] [--scheme plm,hlld,rk3] [--learned]
                                [--layout lean|standard]

Both paths advance the same seeded turbulence box with the same fixed dt (CFL 0.3 of the
FP64 path's primed MaxLambda) and are compared after every `--every` steps: relative L1 and
L-infinity of every primitive field over the interior, the corner divergence of the FP32
path's (FP64) magnetic field, and the failure counts.  Prints one JSON line per checkpoint.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def rel_errors(a, b):
    names = ["rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"]
    A = a[3:-3, 3:-3, 3:-3].reshape(-1, 8)
    B = b[3:-3, 3:-3, 3:-3].reshape(-1, 8)
    l1, linf = {}, {}
    for q, nm in enumerate(names):
        d = np.abs(A[:, q] - B[:, q])
        s1, sinf = np.abs(B[:, q]).mean(), np.abs(B[:, q]).max()
        l1[nm] = float(d.mean() / s1) if s1 > 0 else float(d.mean())
        linf[nm] = float(d.max() / sinf) if sinf > 0 else float(d.max())
    return l1, linf


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--every", type=int, default=25)
    ap.add_argument("--scheme", default="plm,hlld,rk3")
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--layout", default="lean", choices=["lean", "standard"],
                    help="device layout of the FP32 path (the FP64 path is the standard layout)")
    args = ap.parse_args(argv)
    import torch
    from . import ics
    from .mara import Scheme, Solver
    torch.cuda.set_device(0)
    extrap, riemann, advance = args.scheme.split(",")
    n = (args.n,) * 3
    t0 = time.time()
    P0 = ics.turbulence_box(n, seed=args.seed)
    ic_sec = time.time() - t0
    ref = Solver(Scheme(extrap=extrap, riemann=riemann, advance=advance), n)
    fast = Solver(Scheme(extrap=extrap, riemann=riemann, advance=advance, precision="fp32",
                         learned_c2p=args.learned, layout=args.layout), n)
    if args.learned:
        from .train_c2p import load
        fast.set_c2p_network(load())
    for s in (ref, fast):
        s.upload(P0)
        assert s.advance(0.0) == 0
    dt = ref.get_timestep(0.3)
    del P0
    errs = {"fp64": 0, "fp32": 0}
    done = 0
    while done < args.steps:
        k = min(args.every, args.steps - done)
        for key, s in (("fp64", ref), ("fp32", fast)):
            for _ in range(k):
                errs[key] += s.advance(dt)
        done += k
        a, b = fast.download(), ref.download()
        l1, linf = rel_errors(a, b)
        dm, dx = fast.mean_max_divB_state()
        print(json.dumps({"n": args.n, "scheme": args.scheme, "learned": args.learned, "layout": args.layout,
                          "step": done, "dt": dt,
                          "l1_rel": l1, "linf_rel": linf, "divB_fp32": [dm, dx],
                          "failed_zones_total": errs, "ic_seconds": round(ic_sec, 1)}), flush=True)
    ref.close()
    fast.close()


if __name__ == "__main__":
    main()
