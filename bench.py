"""Benchmark: plain mixed-radix + Rader batch, ComplexF64, on B200.

Workload (one step): forward and inverse FFT of a [1024, 30240] batch
(2^5*3^3*5*7, mixed radix) and of a [1024, 10007] batch (prime, Rader), all
ComplexF64 with iid N(0,1) parts (seeded synthetic data), contiguous
[batch][n] layout.  Inputs (1.32 GB) exceed the 126 MB L2, so no flush is
needed between timed iterations.

Metric: FFT GB/s of algorithmic traffic (one read + one write of every
element: 32 B per ComplexF64 element per transform, no extra credit for the
convolution or multi-pass work), reported against the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun every rank runs the same workload on its own GPU (replicas,
no collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
SIZES = [(30240, 1024), (10007, 1024)]
ELEM = 16  # ComplexF64 bytes
METRIC = "FFT GB/s vs HBM peak, plain vs batched/served; p50/p99 latency at stated err"
WORKLOAD = "plain mixed-radix + Rader batch: C128 1024 x n=30240 and 1024 x n=10007, fwd + inv"


def algorithmic_bytes_per_step():
    # fwd + inv of each batch, read + write each element once
    return sum(2 * 2 * n * b * ELEM for n, b in SIZES)


def flops_per_step():
    return sum(2 * b * 5 * n * np.log2(n) for n, b in SIZES)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                out[parts[0]] = float(parts[2])
    return out


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if r[5 + i].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_reference(threads, budget_s, steps=1):
    """Time the oracle (CPU restatement of the reference path) on host cores.

    Each step is a bounded sample: as many whole (fwd+inv of one 30240 and one
    10007 transform) units as fit in budget_s, batched across `threads`.
    Returns (GB/s, seconds, units).
    """
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    rng = np.random.default_rng(1)
    unit_bytes = sum(2 * 2 * n * ELEM for n, _ in SIZES)
    for n, _ in SIZES:
        oracle.prepare(n)
    xs = {n: rng.standard_normal((threads, n)) + 1j * rng.standard_normal((threads, n))
          for n, _ in SIZES}
    vals = []
    for _ in range(steps):
        t0 = time.perf_counter()
        units = 0
        while True:
            for n, _ in SIZES:
                y = oracle.fft(xs[n], threads=threads)
                oracle.ifft(y, threads=threads)
            units += threads
            if time.perf_counter() - t0 > budget_s:
                break
        dt = time.perf_counter() - t0
        vals.append((units * unit_bytes / dt / 1e9, dt, units))
    return vals


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    budget = max(1.0, 60.0 / max(1, args.steps + args.warmup))
    cpu_reference(threads, 0.5, steps=max(0, min(args.warmup, 1)))
    res = cpu_reference(threads, budget, steps=args.steps)
    gbs = statistics.median(v for v, _, _ in res)
    units = sum(u for _, _, u in res)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 4), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.median(dt for _, dt, _ in res), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded iid N(0,1) ComplexF64",
        "config": {"workload": WORKLOAD, "sample": "bounded per step"},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{units} units (fwd+inv of one 30240 and one 10007 transform) "
                                   f"over {args.steps} steps, OpenMP over {threads} threads; "
                                   "the reference is Julia and cannot run here, so its CPU path is "
                                   "the C restatement in oracle/"},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def measure_e2e(torch, cb, lib, plans, bufs, args, world, dev):
    """End to end through the C ABI host entry: pinned host buffers, the copies
    inside the timed region, fwd + inv of both batches per step."""
    host = []
    for (x, _, _), (n, b) in zip(bufs, SIZES):
        hin = torch.empty((b, n), dtype=torch.complex128, pin_memory=True)
        hin.copy_(x.cpu())
        host.append((hin, torch.empty_like(hin)))
    torch.cuda.synchronize()
    vp = ctypes.c_void_p
    for h, (hin, hout) in zip(plans, host):          # warm the staging buffers
        cb.check(lib.cfft_execute_host(h, vp(hin.data_ptr()), vp(hout.data_ptr()), 0))
    steps = max(1, min(3, args.steps))
    te = time.perf_counter()
    for _ in range(steps):
        for h, (hin, hout) in zip(plans, host):
            cb.check(lib.cfft_execute_host(h, vp(hin.data_ptr()), vp(hout.data_ptr()), 0))
            cb.check(lib.cfft_execute_host(h, vp(hout.data_ptr()), vp(hout.data_ptr()), 1))
    e2e_s = (time.perf_counter() - te) / steps
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_s = tt.item()
    # per step: 2 calls per batch, each copies the batch in and out
    io_bytes = sum(2 * n * b * ELEM for n, b in SIZES)
    return {"value": round(world * algorithmic_bytes_per_step() / e2e_s / 1e9, 4), "unit": "GB/s",
            "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes,
            "ms_per_step": round(e2e_s * 1e3, 3),
            "path": "cfft_execute_host (C ABI), pinned host buffers, fwd+inv of each batch"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--only", type=int, default=0, help="restrict to one transform length")
    ap.add_argument("--batch", type=int, default=0, help="override the batch (profiling cases)")
    ap.add_argument("--quick", action="store_true", help="skip the e2e and CPU-baseline legs")
    args = ap.parse_args()
    global SIZES
    if args.only:
        SIZES = [(n, b) for n, b in SIZES if n == args.only] or [(args.only, 1024)]
    if args.batch:
        SIZES = [(n, args.batch) for n, _ in SIZES]
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(3, args.warmup)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _pkg import load
    cb = load()
    lib = cb._lib.LIB

    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    plans, bufs = [], []
    for n, b in SIZES:
        x = torch.complex(torch.randn(b, n, dtype=torch.float64, device=dev, generator=g),
                          torch.randn(b, n, dtype=torch.float64, device=dev, generator=g))
        y = torch.empty_like(x)
        z = torch.empty_like(x)
        h = ctypes.c_void_p()
        cb.check(lib.cfft_plan_create(ctypes.byref(h), n, b, cb.C128, cb.NO_FLAG))
        plans.append(h)
        bufs.append((x, y, z))
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    launches_per_step = sum(2 * lib.cfft_plan_launches(h) for h in plans)

    def step(ev=None):
        for i, (h, (x, y, z)) in enumerate(zip(plans, bufs)):
            if ev is not None:
                ev[i][0].record(stream)
            cb.check(lib.cfft_execute(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), 0, sp))
            if ev is not None:
                ev[i][1].record(stream)
            cb.check(lib.cfft_execute(h, ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(z.data_ptr()), 1, sp))
            if ev is not None:
                ev[i][2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # correctness guard on the benchmarked data: round trip
    for (x, y, z), (n, _) in zip(bufs, SIZES):
        err = (torch.linalg.norm(z - x) / torch.linalg.norm(x)).item()
        assert err < 1e-12, (n, err)

    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in plans]
           for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        t0.record(stream)
        for s in range(args.steps):
            step(evs[s])
        t1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = tt.item()
    ms_step = ms / args.steps
    value = world * algorithmic_bytes_per_step() / (ms_step * 1e-3) / 1e9

    # per-launch kernel time (each cfft_execute of these plans is one launch)
    per = []
    for i, (n, b) in enumerate(SIZES):
        fw = [evs[s][i][0].elapsed_time(evs[s][i][1]) for s in range(args.steps)]
        iv = [evs[s][i][1].elapsed_time(evs[s][i][2]) for s in range(args.steps)]
        per.append((n, b, statistics.mean(fw + iv), sum(fw) + sum(iv)))
    dom = max(per, key=lambda r: r[3])
    n_dom, b_dom, ms_launch, _ = dom
    achieved = 2 * n_dom * b_dom * ELEM / (ms_launch * 1e-3) / 1e9
    peak, peak_kind = load_peaks()
    traffic = load_traffic().get(f"four_c128_n{n_dom}_b{b_dom}")

    e2e = None if args.quick else measure_e2e(torch, cb, lib, plans, bufs, args, world, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.quick:
        threads = os.cpu_count() or 1
        res = cpu_reference(threads, args.cpu_budget, steps=1)[0]
        cpu = {"value": round(res[0], 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"{res[2]} units (fwd+inv of one 30240 and one 10007 transform) in "
                         f"{res[1]:.1f} s, OpenMP over {threads} threads"}

    for h in plans:
        lib.cfft_plan_destroy(h)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded iid N(0,1) ComplexF64 (torch generator), resident in HBM",
            "config": {"workload": WORKLOAD, "batches": [list(s) for s in SIZES],
                       "l2": "inputs 1.32 GB > 126 MB L2, no flush needed",
                       "parallelism": f"replicas x{world}"},
            "gflops": round(world * flops_per_step() / (ms_step * 1e-3) / 1e9, 2),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": f"k_four<double2> n={n_dom} batch={b_dom}",
                         "ms_per_launch": round(ms_launch, 4)},
            "per_size_ms_per_launch": {str(n): round(m, 4) for n, _, m, _ in per},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
