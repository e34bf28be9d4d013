"""Throughput of Mara.advance(buf, dt) with its host copies (mgpu_advance_host).

    python -m ctf_b200.e2e [--n 512] [--steps 3] [--warmup 1] [--scheme plm,hlld,rk3]
                           [--learned] [--slabs -1 0 ...] [--pageable]

The lean FP32-bulk solver advances a seeded turbulence box through the host buffer, as the
reference's drivers call luaC_Mara_advance (Mara/mara.cpp:297-341): every call copies the
whole guarded AoS primitive array in and, when the advance commits, back out.  Each --slabs
setting of the pipelined call (mgpu_set_pipeline: -1 automatic, 0 unpipelined, >= 3 equal
slabs) is timed by the wall clock around the calls and printed as one JSON line:
interior zone-updates/s and ms per call.  The buffer is pinned unless --pageable.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--scheme", default="plm,hlld,rk3")
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--slabs", type=int, nargs="+", default=[-1, 0])
    ap.add_argument("--pageable", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args(argv)
    import torch
    from . import ics
    from .mara import Scheme, Solver
    torch.cuda.set_device(0)
    extrap, riemann, advance = args.scheme.split(",")
    n = (args.n,) * 3
    s = Solver(Scheme(extrap=extrap, riemann=riemann, advance=advance, precision="fp32", layout="lean",
                      learned_c2p=args.learned), n)
    if args.learned:
        from .train_c2p import load
        s.set_c2p_network(load())
    P0 = ics.turbulence_box(n, seed=args.seed)
    if args.pageable:
        host = P0
    else:
        host = torch.empty(P0.size, dtype=torch.float64, pin_memory=True).numpy().reshape(P0.shape)
        host[...] = P0
        del P0
    s.upload(host)
    assert s.advance(0.0) == 0
    dt = 0.5 * s.get_timestep(0.3)   # a fixed dt well inside the CFL limit of every call
    for slabs in args.slabs:
        s.set_pipeline(slabs)
        for _ in range(args.warmup):
            s.advance_host(host, dt)
        torch.cuda.synchronize()
        errors = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            errors += s.advance_host(host, dt)[1]
        sec = (time.perf_counter() - t0) / max(args.steps, 1)
        print(json.dumps({"n": args.n, "scheme": args.scheme, "learned": args.learned,
                          "pinned": not args.pageable, "slabs_setting": slabs, "slabs": s.pipeline()[1],
                          "ms_per_call": sec * 1e3, "zone_updates_per_s": float(np.prod(n)) / sec,
                          "errors": errors}), flush=True)
    s.close()


if __name__ == "__main__":
    main()
