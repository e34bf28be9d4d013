#!/usr/bin/env python
"""Benchmark of the B200 RMHD step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

A step is one full Mara advance (all RK stages) of a seeded synthetic box.  The headline
workload is the 512^3 relativistic-MHD turbulence box (rho = p = 1, Gamma 4/3, Gaussian
random velocity with per-mode power ~ |k|^-2 on 1 <= |k| <= 4, rms 0.3c, |v| < 0.9;
B = (0, 0, 1) + solenoidal perturbation of rms 0.1) with PLM (minmod theta 2) + HLLD + RK3 +
flux-CT, CFL 0.3.  `value` is the FP32-bulk path with the learned c2p guess (FP64 c2p
polish, magnetic field and dt); the plain FP64 path runs the same steps in the same call and
is reported beside it -- both the parity build (every multiply and add rounded separately,
as the reference's x86-64 build does) and the same kernels compiled with fused multiply-add
-- with the relative L1 and Linf difference of every primitive against FP64 after the timed
steps, and the failed zones of the timed steps.

The FP32 runs use the lean device layout by default (`--layout lean`: the sweeps add their
flux differences straight into the Runge-Kutta register, only the transverse face fields are
stored; `--layout standard` for the stored-flux layout); the FP64 runs use the standard
layout, the one held to the reference's golden steps.

`e2e` times the same FP32 + learned solver through Mara.advance(buf, dt) with a pinned host
buffer: every call copies the whole guarded AoS array in and back out.  In the lean layout that
call is pipelined over slabs of x rows (the copies overlap the advance; the result is the
unpipelined call's bit for bit), and `e2e.value_unpipelined` gives the same calls with the
pipeline switched off.

All precisions advance with the same fixed dt (CFL 0.3 of the primed MaxLambda) so their
final states are comparable.  Every array (8.9 GB per FP64 state at 512^3) is larger than
the 126 MB L2, so no flush is needed between steps.  For N > 1 (torchrun) every rank
advances its own box: independent replicas, weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RMHD zone-updates/s on 1 B200: FP32+learned c2p vs plain FP64 at stated L1 err"
UNIT = "zone-updates/s"

WORKLOADS = {
    # name: (n, ic, scheme kwargs)
    "turb256_weno5_hlld_rk3": ((256, 256, 256), "turbulence",
                               dict(extrap="weno5", riemann="hlld", advance="rk3")),
    "turb64_plm_hlld_rk2": ((64, 64, 64), "turbulence", dict(extrap="plm", riemann="hlld", advance="rk2")),
    "turb512_plm_hlld_rk3": ((512, 512, 512), "turbulence",
                             dict(extrap="plm", riemann="hlld", advance="rk3")),
    "turb128_weno5_hlld_rk3": ((128, 128, 128), "turbulence",
                               dict(extrap="weno5", riemann="hlld", advance="rk3")),
    # profiling sizes: the face array (166^3 x 8 x 4 B = 146 MB) still exceeds the 126 MB L2
    "turb160_weno5_hlld_rk3": ((160, 160, 160), "turbulence",
                               dict(extrap="weno5", riemann="hlld", advance="rk3")),
    "turb160_plm_hlld_rk3": ((160, 160, 160), "turbulence",
                             dict(extrap="plm", riemann="hlld", advance="rk3")),
    "turb256_plm_hlld_rk3": ((256, 256, 256), "turbulence",
                             dict(extrap="plm", riemann="hlld", advance="rk3")),
    # the high-magnetisation stress box (W log-uniform in [1, 10], sigma log-uniform in
    # [0.1, 10], p = 0.01): the reference's algorithm fails its first step, so it runs with the
    # reference's emergency reset (config_solver{ereset = true, preset = 0.01, dreset = 1})
    "stress512_plm_hlld_rk3": ((512, 512, 512), "stress",
                               dict(extrap="plm", riemann="hlld", advance="rk3", ereset=True, preset=0.01,
                                    dreset=1.0)),
    "stress128_plm_hlld_rk3": ((128, 128, 128), "stress",
                               dict(extrap="plm", riemann="hlld", advance="rk3", ereset=True, preset=0.01,
                                    dreset=1.0)),
}
DEFAULT_WORKLOAD = "turb512_plm_hlld_rk3"
# ensembles: 256 independent 2D Kelvin-Helmholtz boxes, sides log-uniform in 64..512
ENSEMBLE_WORKLOADS = {
    "kh_ensemble256_plm_hllc_rk3": dict(nboxes=256, lo=64, hi=512,
                                        scheme=dict(extrap="plm", riemann="hllc", advance="rk3")),
}
# large driven boxes in the lean layout (FP32 bulk + learned c2p), OU velocity forcing
# (correlation time 1, forcing power 0.3^2 on 1 <= |k| <= 3), uniform start rho = p = 1,
# B = (0, 0, 0.5), v = 0; the loop of the reference's driven-turbulence driver
# (ctf-core/drvtrb.lua:480-488): advance, OU step of the field, resample every 10 steps
DRIVEN_WORKLOADS = {
    "drive1024_weno5_hlld_rk3": dict(n=(1024, 1024, 1024), power=0.09, k1=3, zeta=1.0, Bz=0.5,
                                     scheme=dict(extrap="weno5", riemann="hlld", advance="rk3")),
    "drive256_weno5_hlld_rk3": dict(n=(256, 256, 256), power=0.09, k1=3, zeta=1.0, Bz=0.5,
                                    scheme=dict(extrap="weno5", riemann="hlld", advance="rk3")),
}
CFL = 0.3

# Figures from ncu captures of the FP32-bulk kernels on a 160^3 box of the same scheme,
# keyed by (kernel class, reconstruction, Riemann solver, layout): DRAM bytes
# (dram__bytes_read.sum + dram__bytes_write.sum) per work unit, and the issue/pipe
# utilisation that bounds the lean HLLD sweeps.  They come from separate captures, not from
# the run that prints them.
NCU_TRAFFIC_PER_UNIT = {("update", "plm", "hlld", "lean"): 69.7,    # a first-stage CT launch
                        # the x sweep's DRAM bytes per zone, 120.2 against its 100 algorithmic,
                        # applied as that 1.202 ratio to the mean of the three sweeps (86.7 B)
                        ("flux", "plm", "hlld", "lean"): 104.2}
NCU_LIMITER = {
    ("flux", "plm", "hlld", "lean"): {"issue_active": 0.507, "fma_pipe": 0.263, "xu_pipe": 0.133,
                                      "dram_throughput": 0.086},
    ("flux", "weno5", "hlld", "lean"): {"issue_active": 0.467, "fma_pipe": 0.281, "xu_pipe": 0.194,
                                        "dram_throughput": 0.068},
    ("flux", "weno5", "hlld", "standard"): {"issue_active": 0.500, "fma_pipe": 0.292, "xu_pipe": 0.210},
}


def make_ic(kind, n, seed=0):
    from ctf_b200 import ics
    if kind == "turbulence":
        return ics.turbulence_box(n, seed=seed)
    if kind == "stress":
        return ics.stress_box(n, seed=seed)
    raise ValueError(kind)


def launches_per_step(nd, rk):
    ns = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}[rk]
    return 2 + ns * (2 + nd) + 2


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()   # sampling is live before the timed region starts
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def time_device(solver, steps, warmup, dt, torch, stream):
    """Warm up, then time `steps` advances with CUDA events on the solver's stream.  Returns
    the milliseconds, the per-class kernel profile of the timed advances and the solver's
    statistics after the warm-up (its cumulative advance counters mark the timed region)."""
    solver.advance_async(warmup, dt=dt)
    solver.synchronize()
    st_warm = solver.stats()
    solver.profile_read()   # drop warm-up launches
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    solver.advance_async(steps, dt=dt)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end)
    prof = solver.profile_read()
    return ms, prof, st_warm


def rel_linf(a, b, nd, ng=3):
    """max |a - b| / max |b| per primitive over the interior zones."""
    sl = tuple(slice(ng, -ng) if d < nd else slice(None) for d in range(3))
    a, b = a[sl], b[sl]
    out = {}
    for q, name in enumerate(["rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"]):
        den = np.abs(b[..., q]).max()
        num = np.abs(a[..., q] - b[..., q]).max()
        out[name] = float(num / den) if den > 0 else float(num)
    return out


def ghost_factor(n_sample, n_workload, ng=3):
    """The reference advances every guarded zone (c2p over all of them, fluxes over almost
    all faces), so its interior zone-updates/s on a small sample box understate its rate on a
    large box by the ratio of the two boxes' guarded-to-interior zone counts."""
    def over(m):
        m = [m] * 3 if np.isscalar(m) else list(m)
        return float(np.prod([(v + 2 * ng) / v for v in m]))
    return over(n_sample) / over(n_workload)


def rel_l1(a, b, nd, ng=3):
    sl = tuple(slice(ng, -ng) if d < nd else slice(None) for d in range(3))
    a, b = a[sl], b[sl]
    out = {}
    for q, name in enumerate(["rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"]):
        den = np.abs(b[..., q]).mean()
        num = np.abs(a[..., q] - b[..., q]).mean()
        out[name] = float(num / den) if den > 0 else float(num)
    return out


def cpu_sample(scheme_kw, steps=2, n=64, use_ref=True, seed=0, warmup=0, ic="turbulence"):
    """Time the reference's CPU advance (or the C restatement) on a bounded sample box, after
    `warmup` untimed advances."""
    from oracle import PortOracle, REF_SO, RefOracle, Scheme
    sch = Scheme(n=(n, n, n), **scheme_kw)
    kind = "reference" if (use_ref and os.path.exists(REF_SO)) else "port"
    o = RefOracle(sch) if kind == "reference" else PortOracle(sch)
    P = make_ic(ic, (n, n, n), seed=seed)
    o.advance(P, 0.0)
    dt = o.get_timestep(CFL)
    for _ in range(warmup):
        o.advance(P, dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.advance(P, dt)
    sec = time.perf_counter() - t0
    if kind == "reference":
        o.close()
    return kind, n ** 3 * steps / sec, sec


def _cpu_worker(args):
    scheme_kw, steps, n, seed, warmup, ic = args
    return cpu_sample(scheme_kw, steps=steps, n=n, seed=seed, warmup=warmup, ic=ic)


def cpu_sample_kh(scheme_kw, steps=2, n=256, seed=0, warmup=0):
    """The reference's CPU advance of one 2D Kelvin-Helmholtz box (bounded sample), after
    `warmup` untimed advances."""
    from ctf_b200 import ics
    from oracle import PortOracle, REF_SO, RefOracle, Scheme
    sch = Scheme(n=(n, n), **scheme_kw)
    kind = "reference" if os.path.exists(REF_SO) else "port"
    o = RefOracle(sch) if kind == "reference" else PortOracle(sch)
    P = np.ascontiguousarray(ics.kh_box((n, n), seed=seed))
    o.advance(P, 0.0)
    dt = o.get_timestep(CFL)
    for _ in range(warmup):
        o.advance(P, dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.advance(P, dt)
    sec = time.perf_counter() - t0
    if kind == "reference":
        o.close()
    return kind, n * n * steps / sec, sec


def _cpu_worker_kh(args):
    scheme_kw, steps, n, seed, warmup = args
    return cpu_sample_kh(scheme_kw, steps=steps, n=n, seed=seed, warmup=warmup)


def run_ensemble_bench(args, rank, world, local):
    """An ensemble of independent 2D KH boxes advanced as one CUDA graph per step (FP32 bulk,
    autotuned launch shape), with the FP64 ensemble of the same boxes and dt beside it."""
    import torch
    from ctf_b200 import ics
    from ctf_b200.ensemble import Ensemble, kh_sizes
    from ctf_b200.mara import Scheme
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    wl = ENSEMBLE_WORKLOADS[args.workload]
    kw = wl["scheme"]
    sizes = kh_sizes(wl["nboxes"], seed=rank, lo=wl["lo"], hi=wl["hi"])
    states = [np.ascontiguousarray(ics.kh_box(n, seed=1000 * rank + b)) for b, n in enumerate(sizes)]
    zones = sum(a * b for a, b in sizes)
    stream = torch.cuda.Stream()

    def make(prec):
        E = Ensemble(Scheme(precision=prec, **kw), sizes)
        E.set_stream(stream.cuda_stream)
        for b, P in enumerate(states):
            E.upload(b, P)
        E.advance(dt=0.0)
        return E

    def timed(E, dt):
        E.advance(dt=dt, nsteps=1)   # capture the one-step graph
        for _ in range(args.warmup - 1):
            E.advance(dt=dt, nsteps=1)
        E.synchronize()
        if dist is not None:
            dist.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            start.record(stream)
            for _ in range(args.steps):
                E.advance(dt=dt, nsteps=1)
            end.record(stream)
            end.synchronize()
        ms = start.elapsed_time(end)
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        assert not E.errors().any(), "an ensemble box failed"
        return ms, clk.summary()

    out_runs, finals = {}, {}
    dt = None
    for prec in (["fp64"] if not args.skip_fp64 else []) + ["fp32"]:
        E = make(prec)
        if dt is None:
            dt = E.timesteps(CFL)
        tune = None
        if prec == "fp32":
            shape, tms = E.autotune(dt, reps=2)
            tune = {"launch": shape, "ms_per_step": tms}
        ms, clk = timed(E, dt)
        finals[prec] = [E.download(b) for b in range(E.nb)]
        # kernel shares from one direct (profiled) advance of the same state
        E.profile_enable(256)
        E.advance(dt=dt, nsteps=1, graph=False)
        prof = E.profile_read()
        E.profile_disable()
        out_runs[prec] = {"value": zones * args.steps * world / (ms * 1e-3), "ms_per_step": ms / args.steps,
                          "clocks": clk, "prof": prof, "tuning": tune, "ensemble": E}
        if prec == "fp64":
            E.close()
    head = out_runs["fp32"]
    E = head["ensemble"]
    prof = head["prof"]
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    dom = max(("flux", "update", "c2p", "p2c"), key=lambda k: prof[k]["ms"])
    per_unit = {"flux": 16 * 4, "update": 5 * 4 * 3 + 3 * 8 * 3 + 2 * 8 * 4, "c2p": 44 + 8 * 4, "p2c": 88}
    d = prof[dom]
    achieved = per_unit[dom] * d["units"] / (d["ms"] * 1e-3) / 1e9
    line = {
        "metric": "RMHD zone-updates/s on 1 B200: ensemble of 256 uneven 2D KH boxes, FP32 bulk, one graph per step",
        "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "boxes": wl["nboxes"], "sides": [wl["lo"], wl["hi"]],
                   "interior_zones": zones, "scheme": kw, "cfl": CFL,
                   "dt": "per box, CFL 0.3 of its primed MaxLambda (same for both precisions)",
                   "l2": "all boxes' arrays together (~4 GB) > 126 MB L2 (no flush needed)",
                   "launch": head["tuning"]["launch"], "tuned_ms_per_step": head["tuning"]["ms_per_step"]},
        "gpu_launches": (2 + 3 * 4 + 2) * args.steps,
        "clocks": head["clocks"],
        "runs": {k: {"value": r["value"], "ms_per_step": r["ms_per_step"],
                     "kernel_ms_per_step": {c: r["prof"][c]["ms"] for c in r["prof"]}}
                 for k, r in out_runs.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes_per_unit": per_unit[dom]},
    }
    if "fp64" in finals:
        line["speedup_vs_fp64"] = head["value"] / out_runs["fp64"]["value"]
        # rho and p relative to themselves; v and B components relative to the mean |v| and
        # |B| of the box (vy, By start as small perturbations of a shear flow along x)
        num = np.zeros(8)
        den = np.zeros(8)
        for a, b in zip(finals["fp32"], finals["fp64"]):
            a, b = a[3:-3, 3:-3].reshape(-1, 8), b[3:-3, 3:-3].reshape(-1, 8)
            vs = np.sqrt((b[:, 2:5] ** 2).sum(1)).sum()
            bs = np.sqrt((b[:, 5:8] ** 2).sum(1)).sum()
            num += np.abs(a - b).sum(0)
            den += np.array([np.abs(b[:, 0]).sum(), np.abs(b[:, 1]).sum(), vs, vs, vs, bs, bs, bs])
        names = ["rho", "pre", "vx", "vy", "vz", "Bx", "By", "Bz"]
        line["l1_rel_vs_fp64"] = {n: float(num[q] / den[q]) for q, n in enumerate(names)}
    if not args.no_e2e:
        hosts = []
        for b, P in enumerate(states):
            h = torch.empty(P.shape, dtype=torch.float64, pin_memory=True).numpy()
            h[...] = E.download(b)
            hosts.append(h)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for b in range(E.nb):
                E.lib.mgpu_ensemble_upload_prim(E.h, b, hosts[b].ctypes.data_as(
                    ctypes.POINTER(ctypes.c_double)))
            E.advance(dt=dt, nsteps=1)
            errs = E.errors()
            for b in range(E.nb):
                E.lib.mgpu_ensemble_download_prim(E.h, b, hosts[b].ctypes.data_as(
                    ctypes.POINTER(ctypes.c_double)))
        sec = time.perf_counter() - t0
        assert not errs.any()
        nbytes = sum(h.nbytes for h in hosts)
        line["e2e"] = {"value": zones * args.steps * world / sec, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes,
                       "api": "mgpu_ensemble_upload_prim + mgpu_ensemble_advance + mgpu_ensemble_download_prim"}
    E.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        kind, v, sec = cpu_sample_kh(kw, steps=2, n=256)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": kind,
                                "sample": f"one 256^2 KH box, same scheme, 2 steps after priming ({sec:.1f} s), "
                                          "interior zone-updates/s on 1 core"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_driven_bench(args, rank, world, local):
    """A large driven box in the lean layout: FP32 bulk + learned c2p, OU driving, as the
    reference's driven-turbulence driver runs it.  The box starts uniform and is filled slab
    by slab (one x-plane of host memory); the timed region is K driver steps (get_timestep,
    advance with its driving kick, OU step of the field, a resample every 10 steps), timed
    with CUDA events on the solver's stream around the whole loop."""
    import torch
    from ctf_b200.mara import Scheme, Solver, new_ou_field
    from ctf_b200.train_c2p import load as load_net
    wl = DRIVEN_WORKLOADS[args.workload]
    n, kw = wl["n"], wl["scheme"]
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    net_path = os.path.join(ROOT, "ctf_b200", "data", "c2p_net.npz")
    learned = os.path.exists(net_path) and not args.no_learned
    s = Solver(Scheme(precision="fp32", layout="lean", learned_c2p=learned, **kw), n, stream=stream.cuda_stream)
    if learned:
        s.set_c2p_network(load_net(net_path))
    G = [m + 6 for m in n]
    plane = np.zeros((G[1] * G[2], 8))
    plane[:, 0] = 1.0
    plane[:, 1] = 1.0
    plane[:, 7] = wl["Bz"]
    t_ic = time.perf_counter()
    for i in range(G[0]):
        s.upload_range(plane, i * G[1] * G[2])
    s.set_driving(new_ou_field(3, wl["power"], wl["zeta"], wl["k1"], 1000 + rank))
    t_ic = time.perf_counter() - t_ic
    assert s.advance(0.0) == 0, "priming advance failed"
    it = [0]

    def driver_step():
        dt = s.get_timestep(CFL)
        e = s.advance(dt)
        if e == 0:
            s.driving_advance(dt)
            if it[0] % 10 == 0:
                s.driving_resample()
        it[0] += 1
        return e

    for _ in range(args.warmup):
        assert driver_step() == 0
    s.profile_enable(capacity=64 * (args.steps + 1))
    s.profile_read()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    errs = 0
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            errs += driver_step()
        end.record(stream)
        end.synchronize()
    ms = start.elapsed_time(end)
    prof = s.profile_read()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    zones = int(np.prod(n))
    st = s.stats()
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    state = 5 * 4 + 3 * 8
    # lean sweeps: read the 8 FP32 stage primitives, write two face fields, read-modify-write
    # the 5 FP32 register components (the x sweep also reads U^n): averaged over x, y, z
    per_unit = {"flux": 32 + 8 + (60 + 40 + 40) / 3.0,
                "update": 3 * 8 * 3 + 6 * 4,       # CT: read U^n.B, U^(s).B, write U.B, read 6 face fields
                "c2p": state + 8 * 4}
    dom = max(("flux", "update", "c2p"), key=lambda k: prof[k]["ms"])
    d = prof[dom]
    alg = per_unit[dom] * d["units"] / max(d["launches"], 1)
    achieved = alg / (d["ms"] / max(d["launches"], 1) * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": zones * args.steps * world / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "n": list(n), "scheme": kw, "cfl": CFL, "layout": "lean",
                   "precision": "fp32 bulk; fp64 c2p polish, magnetic field, CT and dt"
                                + ("; learned c2p guess (bf16 tcgen05 MLP)" if learned else ""),
                   "driving": {k: wl[k] for k in ("power", "k1", "zeta")} | {"resample_every": 10},
                   "ic": f"uniform rho=p=1, Bz={wl['Bz']}, v=0 (driven from rest), {t_ic:.0f} s to fill",
                   "l2": "every state array > 126 MB L2 (no flush needed)",
                   "parallelism": f"{world} independent replica(s)",
                   "device_bytes_per_zone": 144},
        "gpu_launches": int(sum(v["launches"] for v in prof.values())),
        "clocks": clk.summary(), "errors": errs,
        "kernel_ms_per_step": {k: v["ms"] / args.steps for k, v in prof.items()},
        "c2p_iters_per_call": st["c2p_iters"] / max(st["c2p_calls"], 1),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "algorithmic_bytes_per_unit": per_unit[dom],
                     "kernel_share": {k: v["ms"] / sum(x["ms"] for x in prof.values()) for k, v in prof.items()}},
        "e2e": None,
        "e2e_note": "not measured for this workload: the AoS host buffer of a 1030^3 box is 70 GB per direction",
    }
    s.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        kind, v, sec = cpu_sample(kw, steps=2, n=48)
        corr = ghost_factor(48, n)
        out["cpu_baseline"] = {"value": v * corr, "unit": UNIT, "cores": 1, "kind": kind,
                               "measured_value": v, "ghost_correction": corr,
                               "sample": f"48^3 turbulence box, same scheme (undriven), 2 steps after priming "
                                         f"({sec:.1f} s), interior zone-updates/s on 1 core; value = measured x "
                                         f"{corr:.3f} (guarded-to-interior zone ratio of the sample over that of "
                                         f"the workload)"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def tiled_block(tile: np.ndarray, off, n, ng=3) -> np.ndarray:
    """The guarded block [off - ng, off + n + ng) of the periodic box made by repeating the
    interior of `tile` (a guarded turbulence box) along every axis: a large periodic state
    whose blocks each rank builds on its own, without the global array."""
    t = tile[ng:-ng, ng:-ng, ng:-ng]
    idx = [np.arange(o - ng, o + m + ng) % t.shape[d] for d, (o, m) in enumerate(zip(off, n))]
    return np.ascontiguousarray(t[np.ix_(*idx)])


def run_decomposed_bench(args, rank, world, local):
    """--decompose: one box of the workload split over the ranks (DecomposedSolver, standard
    layout, FP32 bulk + learned c2p as the headline run), the guard exchange of every RK stage
    over NCCL overlapped with the cores' c2p: strong scaling.  The state is a 128^3 turbulence
    box repeated periodically to the workload's size (each rank builds only its block)."""
    import torch
    from ctf_b200 import ics
    from ctf_b200.decomp import DecomposedSolver, Layout, TorchTransport, rank_dims
    from ctf_b200.mara import Scheme
    dist = None
    torch.cuda.set_device(local if world > 1 else 0)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    n, _, scheme_kw = WORKLOADS[args.workload]
    net_path = os.path.join(ROOT, "ctf_b200", "data", "c2p_net.npz")
    learned = os.path.exists(net_path) and not args.no_learned
    scheme = Scheme(precision="fp32", learned_c2p=learned, **scheme_kw)
    dims = rank_dims(world, 3, n)
    L = Layout(N=n, dims=dims, x0=(0.0,) * 3, x1=(1.0,) * 3)
    D = DecomposedSolver(scheme, L, ranks=[rank], transport=TorchTransport(dist) if dist else None)
    if learned:
        from ctf_b200.train_c2p import load as load_net
        for b in D.blocks:
            b.solver.set_c2p_network(load_net(net_path))
    tile = ics.turbulence_box((128, 128, 128), seed=0)
    for b in D.blocks:
        b.solver.upload(tiled_block(tile, b.off, b.n))
    D.advance(dt=0.0)
    assert D.errors() == 0, "priming advance failed"
    dt = D.get_timestep(CFL)
    for _ in range(args.warmup):
        D.advance(dt=dt)
    D.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(D.stream)
        for _ in range(args.steps):
            D.advance(dt=dt)
        end.record(D.stream)
        end.synchronize()
    ms = start.elapsed_time(end)
    errs = D.errors()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    zones = int(np.prod(n))
    nst = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}[scheme_kw["advance"]]
    # per advance: begin + per stage (shell c2p, core c2p, 3 sweeps, update) + closing c2p +
    # commit, plus 4 slab pack/unpack kernels per split dimension and stage
    per_adv = 2 + nst * (2 + 3 + 1) + 1 + nst * 4 * len(L.split())
    out = {"metric": METRIC, "value": zones * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": args.workload, "n": list(n), "scheme": scheme_kw, "cfl": CFL, "dt": dt,
                      "layout": "standard", "decomposition": list(dims),
                      "precision": "fp32 bulk; fp64 c2p polish, magnetic field, CT and dt"
                                   + ("; learned c2p guess" if learned else ""),
                      "ic": "128^3 turbulence box repeated periodically",
                      "exchange": "NCCL point-to-point per RK stage, overlapped with the cores' c2p",
                      "l2": "every state array > 126 MB L2 (no flush needed)",
                      "parallelism": f"{world} ranks, one box"},
           "gpu_launches": per_adv * args.steps, "clocks": clk.summary(), "errors": errs,
           "e2e": None, "e2e_note": "the decomposed mode keeps the state on the devices (no host copies)"}
    D.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_reference_arm(args, wl_name, rank, world):
    """--impl reference: the reference's own CPU advance on every host core (independent
    replicas of a 64^3 sample box of the workload's scheme, or 256^2 KH boxes for an
    ensemble workload)."""
    if rank != 0:
        return
    if wl_name in ENSEMBLE_WORKLOADS:
        import multiprocessing as mp
        kw = ENSEMBLE_WORKLOADS[wl_name]["scheme"]
        cores = os.cpu_count() or 1
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(cores) as pool:
            res = pool.map(_cpu_worker_kh, [(kw, args.steps, 256, s, args.warmup) for s in range(cores)])
        wall = time.perf_counter() - t0
        value = float(sum(r[1] for r in res))
        line = {"metric": "RMHD zone-updates/s on 1 B200: ensemble of 256 uneven 2D KH boxes, FP32 bulk, "
                          "one graph per step", "value": value, "unit": UNIT, "impl": "reference",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": float(np.mean([r[2] for r in res]) / args.steps * 1e3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": wl_name, "sample": f"{cores} replicas of a 256^2 KH box"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": res[0][0],
                                 "sample": f"{cores} concurrent 256^2 KH boxes x {args.steps} steps; wall {wall:.1f} s"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    ic = "turbulence"
    if wl_name in DRIVEN_WORKLOADS:
        n_wl, scheme_kw = DRIVEN_WORKLOADS[wl_name]["n"], DRIVEN_WORKLOADS[wl_name]["scheme"]
    else:
        n_wl, ic, scheme_kw = WORKLOADS[wl_name]
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    n = 64 if n_wl[0] >= 64 else n_wl[0]
    steps = args.steps
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(scheme_kw, steps, n, s, args.warmup, ic) for s in range(cores)])
    wall = time.perf_counter() - t0
    kind = res[0][0]
    measured = float(sum(r[1] for r in res))
    corr = ghost_factor(n, n_wl)
    value = measured * corr
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": float(np.mean([r[2] for r in res]) / steps * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": wl_name, "sample": f"{cores} replicas of a {n}^3 box, same scheme",
                   "scheme": scheme_kw, "cfl": CFL},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "measured_value": measured, "ghost_correction": corr,
                         "sample": f"{cores} concurrent replicas x {steps} steps of a {n}^3 {ic} "
                                   f"box ({scheme_kw}), interior zone-updates/s summed; wall {wall:.1f} s; "
                                   f"value = measured x {corr:.3f}, the ratio of guarded to interior zones "
                                   f"of the sample to that of the {n_wl[0]}^3 workload (the reference "
                                   f"advances every guard zone)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(WORKLOADS) + sorted(ENSEMBLE_WORKLOADS) + sorted(DRIVEN_WORKLOADS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-fp64-fmad", action="store_true",
                    help="leave out the comparator run of the FP64 kernels compiled with FMA contraction")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--decompose", action="store_true",
                    help="split one box of the workload over the ranks (strong scaling) instead of "
                         "advancing one box per rank (weak scaling)")
    ap.add_argument("--layout", default="lean", choices=["standard", "lean"],
                    help="device layout of the FP32 runs of the turbulence workloads (lean: 3D, 144 B per "
                         "zone in FP32; the FP64 run always uses the standard layout)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, args.workload, rank, world)
        return
    if args.workload in ENSEMBLE_WORKLOADS:
        run_ensemble_bench(args, rank, world, local)
        return
    if args.workload in DRIVEN_WORKLOADS:
        run_driven_bench(args, rank, world, local)
        return
    if args.decompose:
        run_decomposed_bench(args, rank, world, local)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)

    from ctf_b200.mara import Scheme, Solver

    n, ic_kind, scheme_kw = WORKLOADS[args.workload]
    P0 = make_ic(ic_kind, n, seed=rank)
    stream = torch.cuda.Stream()
    net = None
    net_path = os.path.join(ROOT, "ctf_b200", "data", "c2p_net.npz")
    if os.path.exists(net_path) and not args.no_learned:
        from ctf_b200.train_c2p import load as load_net
        net = load_net(net_path)
    # (key, precision, learned, library variant): FP64 first -- its primed MaxLambda sets the
    # dt all runs share
    runs = []
    if not args.skip_fp64:
        runs.append(("fp64", "fp64", False, ""))
        if not args.skip_fp64_fmad:
            runs.append(("fp64_fmad", "fp64", False, "fmad"))
    runs.append(("fp32", "fp32", False, ""))
    if net is not None:
        runs.append(("fp32+learned", "fp32", True, ""))
    results, states, solvers = {}, {}, {}
    dt_fixed = None
    head_key = "fp32+learned" if net is not None else "fp32"
    zones = int(np.prod(n))
    for key, prec, learned, variant in runs:
        layout = args.layout if prec == "fp32" else "standard"
        s = Solver(Scheme(precision=prec, learned_c2p=learned, layout=layout, **scheme_kw), n,
                   stream=stream.cuda_stream, lib_variant=variant)
        if learned:
            s.set_c2p_network(net)
        s.upload(P0)
        assert s.advance(0.0) == 0, "priming advance failed"
        if dt_fixed is None:
            dt_fixed = s.get_timestep(CFL)
        s.upload(P0)
        s.profile_enable(capacity=launches_per_step(len(n), scheme_kw["advance"]) * (args.steps + args.warmup) + 64)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ms, prof, st_warm = time_device(s, args.steps, args.warmup, dt_fixed, torch, stream)
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        st = s.stats()
        results[key] = {"ms_total": ms, "ms_per_step": ms / args.steps,
                        "value": zones * args.steps * world / (ms * 1e-3), "prof": prof, "stats": st,
                        "clocks": clk.summary(),
                        # the timed steps only (the counters are cumulative since set-up)
                        "advances": st["advances"] - st_warm["advances"],
                        "failed_advances": st["failed_advances"] - st_warm["failed_advances"],
                        "errors": st["failed_zones"] - st_warm["failed_zones"]}
        # compare against the FP64 run as soon as a run ends, keeping only the FP64 state (a
        # 512^3 state is 8.9 GB of host memory per rank)
        fin = s.download()
        if key == "fp64":
            states["fp64"] = fin
        elif "fp64" in states:
            results[key]["l1_rel_vs_fp64"] = rel_l1(fin, states["fp64"], len(n))
            results[key]["linf_rel_vs_fp64"] = rel_linf(fin, states["fp64"], len(n))
        del fin
        s.profile_disable()
        if key == head_key:
            solvers[key] = s
        else:
            s.close()   # one solver on the device at a time (512^3 FP64 alone holds 71 GB)
    solver_fp32 = solvers[head_key]

    head = results[head_key]
    out = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "n": list(n), "scheme": scheme_kw, "cfl": CFL,
                   "layout": f"{args.layout} (FP32 runs); standard (FP64 runs)",
                   "precision": "fp32 bulk; fp64 c2p polish, magnetic field, CT and dt"
                                + ("; learned c2p guess (bf16 tcgen05 MLP)" if head_key.endswith("learned") else ""),
                   "dt": dt_fixed, "l2": "every state array > 126 MB L2 (no flush needed)",
                   "parallelism": f"{world} independent replica(s)"},
        "gpu_launches": int(sum(v["launches"] for v in results[head_key]["prof"].values())),
        "clocks": head["clocks"],
        # failed zones summed over the timed steps of the headline run (Mara.advance's count;
        # a step that fails is not committed)
        "errors": head["errors"], "failed_steps": head["failed_advances"],
    }

    def c2p_it(k):
        st = results[k]["stats"]
        return st["c2p_iters"] / max(st["c2p_calls"], 1)
    out["runs"] = {k: {"value": r["value"], "ms_per_step": r["ms_per_step"],
                       "c2p_iters_per_call": c2p_it(k), "errors": r["errors"],
                       # zone c2p calls that failed every rung of the ladder (with the
                       # emergency reset these are the resets), per call, last advance
                       "c2p_failed_per_call": r["stats"]["c2p_failed"] / max(r["stats"]["c2p_calls"], 1),
                       "c2p_attempt": r["stats"]["c2p_attempt"],
                       "failed_steps": r["failed_advances"],
                       "kernel_ms_per_step": {c: r["prof"][c]["ms"] / args.steps for c in r["prof"]}}
                   for k, r in results.items()}
    if "fp64" in results:
        out["fp64_plain"] = {"value": results["fp64"]["value"], "ms_per_step": results["fp64"]["ms_per_step"],
                             "clocks": results["fp64"]["clocks"],
                             "build": "--fmad=false: every multiply and add rounded as the reference's build does"}
        out["speedup_vs_fp64"] = head["value"] / results["fp64"]["value"]
        out["l1_rel_vs_fp64"] = results[head_key]["l1_rel_vs_fp64"]
        out["linf_rel_vs_fp64"] = results[head_key]["linf_rel_vs_fp64"]
        if "fp32" in results and head_key != "fp32":
            out["runs"]["fp32"]["l1_rel_vs_fp64"] = results["fp32"]["l1_rel_vs_fp64"]
        if "fp64_fmad" in results:
            f = results["fp64_fmad"]
            out["fp64_fmad"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "clocks": f["clocks"],
                                "build": "the same FP64 kernels compiled with FMA contraction (not the parity path)",
                                "linf_rel_vs_fp64": f["linf_rel_vs_fp64"]}
            out["speedup_vs_fp64_fmad"] = head["value"] / f["value"]

    states.clear()   # host memory for the e2e buffers

    # roofline of the dominant kernel (event-timed inside the timed region)
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    hbm = peaks.get("hbm_gbs", 6650.0)
    prof = head["prof"]
    dom = max(("flux", "update", "c2p", "p2c"), key=lambda k: prof[k]["ms"])
    tsz = 4
    nd = len(n)
    ns = {"single": 1, "rk2": 2, "rk3": 3, "rk4": 4}[scheme_kw["advance"]]
    state = 5 * tsz + 3 * 8                             # 44 B: FP32 bulk + FP64 B
    # update: read U^n (+ U^(s) after the first stage), the nd fluxes; write the new state --
    # averaged over the stages (RK4's K registers are not counted)
    upd = (state * (2 * ns + (ns - 1)) + ns * nd * 8 * tsz) / ns
    per_unit = {"flux": 16 * tsz,                       # read 8 face-state comps, write 8 flux comps
                "update": upd,
                "c2p": state + 8 * tsz,                 # read U, write 8 prim comps (interior)
                "p2c": 2 * state}
    if args.layout == "lean":
        # a lean sweep per interior zone: read 8 stage primitives, write 2 face fields, read-modify-
        # write 5 register components (the x sweep also reads U^n); CT reads U^n.B, U^(s).B and six
        # face fields, writes U.B
        per_unit["flux"] = 8 * tsz + 2 * tsz + (3 * 5 * tsz + 2 * (2 * 5 * tsz)) / 3.0
        per_unit["update"] = 3 * 3 * 8 + 6 * tsz
    d = prof[dom]
    alg_bytes_per_launch = per_unit[dom] * d["units"] / max(d["launches"], 1)
    avg_ms = d["ms"] / max(d["launches"], 1)
    achieved = alg_bytes_per_launch / (avg_ms * 1e-3) / 1e9
    # DRAM bytes per work unit (face for the standard flux kernel, interior zone otherwise)
    # from one ncu capture of the same kernel on a 160^3 box of the same scheme -- not this
    # run -- scaled to this launch's units (lean sweeps: the mean of the x, y and z sweeps)
    measured = {("flux", "weno5", "hlld", "standard"): 80.0, ("update", "weno5", "hlld", "standard"): 219.8,
                ("flux", "weno5", "hlld", "lean"): 105.1}
    measured.update(NCU_TRAFFIC_PER_UNIT)
    tpu = measured.get((dom, scheme_kw["extrap"], scheme_kw["riemann"], args.layout)) \
        if head_key.startswith("fp32") else None
    traffic = tpu * d["units"] / max(d["launches"], 1) if tpu else None
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                       "frac": achieved / hbm, "traffic": traffic,
                       "traffic_source": ("ncu dram__bytes_read+write per unit of the same kernel on a 160^3 box "
                                          "of this scheme (a separate capture, not this run), scaled") if tpu else None,
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                       "kernel_share": {k: prof[k]["ms"] / sum(v["ms"] for v in prof.values()) for k in prof},
                       "algorithmic_bytes_per_unit": per_unit[dom]}
    # What bounds the FP32 HLLD sweeps instead of HBM: instruction issue and latency of the
    # ~10^3-operation face (ncu figures of the same kernel on a 160^3 box of the same scheme,
    # from a separate capture, not this run)
    lim = NCU_LIMITER.get((dom, scheme_kw["extrap"], scheme_kw["riemann"], args.layout)) \
        if head_key.startswith("fp32") else None
    if lim:
        out["roofline"]["limiter"] = {"kind": "instruction issue / latency (FP32 pipes)", **lim,
                                      "source": "ncu capture of the same kernel on a 160^3 box, not this run"}
    # The whole step against HBM: the compulsory state-vector transfers of one zone-update
    # (single 2, RK2 5, RK3 8: each stage reads its register(s) and writes one) times the bytes
    # of a state vector (64 B FP64; 44 B FP32 bulk with the FP64 field), at the headline rate
    # of one GPU.
    transfers = {"single": 2, "rk2": 5, "rk3": 8}.get(scheme_kw["advance"])
    if transfers:
        bpz = transfers * (44 if head_key.startswith("fp32") else 64)
        step_gbs = out["value"] / world * bpz / 1e9
        out["step_roofline"] = {"bytes_per_zone_update": bpz, "achieved": step_gbs, "peak": hbm,
                                "unit": "GB/s", "frac": step_gbs / hbm}
    # every kernel class against the HBM roofline (algorithmic bytes / event-timed duration)
    out["kernels"] = {}
    for k in ("flux", "update", "c2p", "p2c"):
        pk = prof[k]
        if pk["launches"] and pk["ms"] > 0:
            gbs = per_unit[k] * pk["units"] / (pk["ms"] * 1e-3) / 1e9
            out["kernels"][k] = {"ms_per_launch": pk["ms"] / pk["launches"], "bytes_per_unit": per_unit[k],
                                 "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / hbm}
    out["c2p_stats"] = {k: head["stats"][k] for k in ("c2p_calls", "c2p_iters", "c2p_attempt", "c2p_failed",
                                                      "face_c2p_calls", "face_c2p_iters", "hlld_ok", "hlld_hllc",
                                                      "pcm_retry")}

    # end to end through Mara.advance(buf, dt) semantics with pinned host buffers
    if not args.no_e2e:
        import torch as _t
        host = _t.empty(solver_fp32.shape, dtype=_t.float64, pin_memory=True).numpy()
        host[...] = P0
        for _ in range(max(1, args.warmup)):
            solver_fp32.advance_host(host, dt_fixed)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e2e_err = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dt = solver_fp32.get_timestep(CFL)
            _, e = solver_fp32.advance_host(host, min(dt, dt_fixed))
            e2e_err += e
        sec = time.perf_counter() - t0
        slabs = solver_fp32.pipeline()[1]
        # the same calls with the slab pipeline switched off, for the record
        solver_fp32.set_pipeline(0)
        t1 = time.perf_counter()
        for _ in range(args.steps):
            dt = solver_fp32.get_timestep(CFL)
            _, e = solver_fp32.advance_host(host, min(dt, dt_fixed))
            e2e_err += e
        sec_plain = time.perf_counter() - t1
        solver_fp32.set_pipeline(-1)
        if dist is not None:
            t = torch.tensor([sec, sec_plain], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec, sec_plain = float(t[0].item()), float(t[1].item())
        nbytes = int(np.prod(solver_fp32.shape)) * 8
        out["e2e"] = {"value": int(np.prod(n)) * args.steps * world / sec, "unit": UNIT,
                      "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "errors": e2e_err,
                      "api": "mgpu_advance_host (Mara.advance(buf, dt)) + mgpu_get_timestep",
                      "pipeline_slabs": slabs,
                      "value_unpipelined": int(np.prod(n)) * args.steps * world / sec_plain}
    solver_fp32.close()

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ns_cpu = 48
        kind, v, sec = cpu_sample(scheme_kw, steps=2, n=ns_cpu, ic=ic_kind)
        corr = ghost_factor(ns_cpu, n)
        out["cpu_baseline"] = {"value": v * corr, "unit": UNIT, "cores": 1, "kind": kind,
                               "measured_value": v, "ghost_correction": corr,
                               "sample": f"{ns_cpu}^3 {ic_kind} box, same scheme, 2 steps after priming "
                                         f"({sec:.1f} s), interior zone-updates/s on 1 core; value = measured x "
                                         f"{corr:.3f}, the ratio of guarded to interior zones of the sample to that "
                                         f"of the {n[0]}^3 workload (the reference advances every guard zone)"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
