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


def load_package():
    """The product package, through its own by-path loader."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "catabra_b200_load", os.path.join(ROOT, "catabrafft.jl_b200", "_load.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.load()


SIZES = [(30240, 1024), (10007, 1024)]
ELEM = 16  # ComplexF64 bytes
METRIC = "FFT GB/s vs HBM peak, plain vs batched/served; p50/p99 latency at stated err"
WORKLOAD = "plain mixed-radix + Rader batch: C128 1024 x n=30240 and 1024 x n=10007, fwd + inv"


def algorithmic_bytes_per_step():
    # fwd + inv of each batch, read + write each element once
    return sum(2 * 2 * n * b * ELEM for n, b in SIZES)


def flops_per_step():
    return sum(2 * b * 5 * n * np.log2(n) for n, b in SIZES)


def max_over_ranks(torch, value, device):
    """The largest of every rank's value (device-timed milliseconds): the
    replicas' job time is the slowest rank's."""
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.item()


def job_gbs(world, bytes_per_rank_step, ms_step):
    """Whole-job throughput of `world` replicas: every rank moves the same
    bytes per step, the step takes the slowest rank's time."""
    return world * bytes_per_rank_step / (ms_step * 1e-3) / 1e9


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
    budget = max(0.05, args.ref_seconds / max(1, args.steps + args.warmup))   # the whole arm: about a minute
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
        host.append((hin, torch.empty((b, n), dtype=torch.complex128, pin_memory=True)))
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
        e2e_s = max_over_ranks(torch, e2e_s, dev)
    # the same through pageable host memory (a Julia Vector, a numpy array):
    # the library stages it through pinned buffers
    pag = [(np.ascontiguousarray(hin.numpy()), np.empty(hin.shape, dtype=np.complex128)) for hin, _ in host]
    for h, (pin, pout) in zip(plans, pag):
        cb.check(lib.cfft_execute_host(h, vp(pin.ctypes.data), vp(pout.ctypes.data), 0))
    tp = time.perf_counter()
    for _ in range(steps):
        for h, (pin, pout) in zip(plans, pag):
            cb.check(lib.cfft_execute_host(h, vp(pin.ctypes.data), vp(pout.ctypes.data), 0))
            cb.check(lib.cfft_execute_host(h, vp(pout.ctypes.data), vp(pout.ctypes.data), 1))
    pag_s = (time.perf_counter() - tp) / steps
    if world > 1:
        pag_s = max_over_ranks(torch, pag_s, dev)
    # per step: 2 calls per batch, each copies the batch in and out
    io_bytes = sum(2 * n * b * ELEM for n, b in SIZES)
    return {"value": round(world * algorithmic_bytes_per_step() / e2e_s / 1e9, 4), "unit": "GB/s",
            "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes,
            "ms_per_step": round(e2e_s * 1e3, 3),
            "path": "cfft_execute_host (C ABI), pinned host buffers, fwd+inv of each batch",
            "pageable": {"value": round(world * algorithmic_bytes_per_step() / pag_s / 1e9, 4), "unit": "GB/s",
                         "ms_per_step": round(pag_s * 1e3, 3)}}


# ---------------------------------------------------------------- other forms
FORMS = ("plain", "small", "precision", "pow2", "batch", "serve")


def _setup_single():
    import torch
    rank, world, local = dist_env()
    if rank != 0:
        return None
    torch.cuda.set_device(local)
    cb = load_package()
    return torch, cb, cb._lib.LIB, torch.device("cuda", local)


def _pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q * (len(v) - 1))))]


def form_small(torch, cb, lib, dev, args):
    """1 x n=4096 ComplexF64: latency of one forward call."""
    n = 4096
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    x = torch.complex(torch.randn(1, n, dtype=torch.float64, device=dev, generator=g),
                      torch.randn(1, n, dtype=torch.float64, device=dev, generator=g))
    y, z = torch.empty_like(x), torch.empty_like(x)
    h = ctypes.c_void_p()
    cb.check(lib.cfft_plan_create(ctypes.byref(h), n, 1, cb.C128, cb.NO_FLAG))
    st = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(st.cuda_stream)
    vp = ctypes.c_void_p
    steps = max(args.steps, 200)
    for _ in range(args.warmup + 10):
        lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
        lib.cfft_execute(h, vp(y.data_ptr()), vp(z.data_ptr()), 1, sp)
    torch.cuda.synchronize()
    err = (torch.linalg.norm(z - x) / torch.linalg.norm(x)).item()
    dev_us, host_us = [], []
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(steps):
        t0 = time.perf_counter()
        a.record(st)
        lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
        b.record(st)
        b.synchronize()
        host_us.append((time.perf_counter() - t0) * 1e6)
        dev_us.append(a.elapsed_time(b) * 1e3)
    # through the host entry: pinned 64 KiB in and out
    hin = torch.empty((1, n), dtype=torch.complex128, pin_memory=True)
    hin.copy_(x.cpu())
    hout = torch.empty((1, n), dtype=torch.complex128, pin_memory=True)
    e2e = []
    for i in range(steps + 10):
        t0 = time.perf_counter()
        cb.check(lib.cfft_execute_host(h, vp(hin.data_ptr()), vp(hout.data_ptr()), 0))
        if i >= 10:
            e2e.append((time.perf_counter() - t0) * 1e6)
    lib.cfft_plan_destroy(h)
    return {"form": "small", "metric": "latency of one 4096-point ComplexF64 forward FFT",
            "value": round(statistics.median(dev_us), 2), "unit": "us", "higher_is_better": False,
            "p50_us": round(_pct(dev_us, 0.5), 2), "p99_us": round(_pct(dev_us, 0.99), 2),
            "host_call_us_p50": round(_pct(host_us, 0.5), 2),
            "e2e": {"value": round(statistics.median(e2e), 2), "unit": "us",
                    "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 16 * n,
                    "path": "cfft_execute_host, pinned host buffers"},
            "roundtrip_rel_l2": err, "steps": steps, "dtype": "f64",
            "config": {"workload": "1 x n=4096 C128, iid N(0,1)"}}


def form_precision(torch, cb, lib, dev, args):
    """ComplexF32 arithmetic with FP64-generated twiddles: 4096 x 2^16 and
    4096 x 3^9, uniform(-1,1) parts; error vs this library's ComplexF64 path
    (itself held to 1e-12 of the oracle by the tests)."""
    sizes = [(65536, args.batch or 4096), (19683, args.batch or 4096)]
    if args.only:
        sizes = [(n, b) for n, b in sizes if n == args.only]
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    st = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(st.cuda_stream)
    vp = ctypes.c_void_p
    out = {}
    total_bytes, total_ms = 0, 0.0
    for n, b in sizes:
        x = torch.complex(torch.rand(b, n, device=dev, generator=g) * 2 - 1,
                          torch.rand(b, n, device=dev, generator=g) * 2 - 1)
        y, z = torch.empty_like(x), torch.empty_like(x)
        h = ctypes.c_void_p()
        cb.check(lib.cfft_plan_create(ctypes.byref(h), n, b, cb.C64, cb.NO_FLAG))
        for _ in range(args.warmup):
            lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
            lib.cfft_execute(h, vp(y.data_ptr()), vp(z.data_ptr()), 1, sp)
        steps = max(3, min(args.steps, 50))
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(steps):
            lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
            lib.cfft_execute(h, vp(y.data_ptr()), vp(z.data_ptr()), 1, sp)
        e.record(st)
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / (2 * steps)
        rows = 64
        xd = x[:rows].to(torch.complex128)
        yd = torch.empty_like(xd)
        h2 = ctypes.c_void_p()
        cb.check(lib.cfft_plan_create(ctypes.byref(h2), n, rows, cb.C128, cb.NO_FLAG))
        lib.cfft_execute(h2, vp(xd.data_ptr()), vp(yd.data_ptr()), 0, sp)
        torch.cuda.synchronize()
        rel = (torch.linalg.norm(y[:rows].to(torch.complex128) - yd) / torch.linalg.norm(yd)).item()
        rt = (torch.linalg.norm(z - x) / torch.linalg.norm(x)).item()
        desc = ctypes.create_string_buffer(256)
        lib.cfft_plan_describe(h, desc, 256)
        lib.cfft_plan_destroy(h)
        lib.cfft_plan_destroy(h2)
        nbytes = 2 * n * b * 8
        out[str(n)] = {"ms_per_launch": round(ms, 4), "GB_s": round(nbytes / (ms * 1e-3) / 1e9, 2),
                       "rel_l2_vs_f64": rel, "roundtrip_rel_l2": rt, "plan": desc.value.decode()}
        total_bytes += nbytes
        total_ms += ms
        del x, y, z
        torch.cuda.empty_cache()
    peak, kind = load_peaks()
    v = total_bytes / (total_ms * 1e-3) / 1e9
    return {"form": "precision", "metric": "FFT GB/s, ComplexF32 with FP64 twiddles",
            "value": round(v, 2), "unit": "GB/s", "higher_is_better": True, "per_size": out,
            "frac_of_hbm": round(v / peak, 4), "peak": peak, "peak_kind": kind, "dtype": "f32",
            "tolerance": 1e-5,
            "config": {"workload": "C64 4096 x 2^16 and 4096 x 3^9, uniform(-1,1), forward"}}


def form_pow2(torch, cb, lib, dev, args):
    """Plain ComplexF64 path on batched power-of-two lengths 2^12 .. 2^22,
    1 GiB of input per size (beyond L2), iid N(0,1) parts; forward and
    inverse per step.  GB/s against the HBM roofline and GFLOP/s in the
    5 N log2 N convention, with torch.fft (cuFFT) on the same batch for
    context."""
    g = torch.Generator(device=dev)
    g.manual_seed(13)
    st = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(st.cuda_stream)
    vp = ctypes.c_void_p
    peak, kind = load_peaks()
    flag = {"none": cb.NO_FLAG, "measure": cb.MEASURE}[args.flag]
    exps = [int(e) for e in args.exps.split(",")] if args.exps else list(range(12, 23))
    out = {}
    total_bytes, total_ms = 0, 0.0
    for k in exps:
        n = 1 << k
        b = args.batch or max(1, (1 << 30) // (16 * n))
        x = torch.complex(torch.randn(b, n, dtype=torch.float64, device=dev, generator=g),
                          torch.randn(b, n, dtype=torch.float64, device=dev, generator=g))
        y, z = torch.empty_like(x), torch.empty_like(x)
        h = ctypes.c_void_p()
        cb.check(lib.cfft_plan_create(ctypes.byref(h), n, b, cb.C128, flag))
        for _ in range(max(3, args.warmup)):
            lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
            lib.cfft_execute(h, vp(y.data_ptr()), vp(z.data_ptr()), 1, sp)
        steps = max(3, min(args.steps, 20))
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(steps):
            lib.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), 0, sp)
            lib.cfft_execute(h, vp(y.data_ptr()), vp(z.data_ptr()), 1, sp)
        e.record(st)
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / (2 * steps)
        rt = (torch.linalg.norm(z - x) / torch.linalg.norm(x)).item()
        # correctness gate at the measured batch: the round trip, and the
        # forward transform of the first and last rows against cuFFT (a
        # forward-only error would cancel in the round trip)
        ref = torch.fft.fft(x[[0, b - 1]], dim=1)
        fwd_err = (torch.linalg.norm(y[[0, b - 1]] - ref) / torch.linalg.norm(ref)).item()
        assert rt < 1e-12 and fwd_err < 1e-12, (n, rt, fwd_err)
        desc = ctypes.create_string_buffer(256)
        lib.cfft_plan_describe(h, desc, 256)
        lib.cfft_plan_destroy(h)
        # cuFFT on the same batch, forward only (context)
        for _ in range(3):
            torch.fft.fft(x, dim=1)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(steps):
            torch.fft.fft(x, dim=1)
        e.record(st)
        torch.cuda.synchronize()
        lib_ms = a.elapsed_time(e) / steps
        nbytes = 2 * n * b * 16
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[str(n)] = {"batch": b, "ms_per_launch": round(ms, 4), "GB_s": round(gbs, 2),
                       "frac_of_hbm": round(gbs / peak, 4),
                       "GFLOP_s": round(5 * n * k * b / (ms * 1e-3) / 1e9, 1),
                       "cufft_ms": round(lib_ms, 4), "roundtrip_rel_l2": rt, "fwd_rel_l2_vs_cufft": fwd_err,
                       "plan": desc.value.decode()}
        total_bytes += nbytes
        total_ms += ms
        del x, y, z
        torch.cuda.empty_cache()
    v = total_bytes / (total_ms * 1e-3) / 1e9
    return {"form": "pow2", "metric": "FFT GB/s vs HBM peak, ComplexF64, batched power-of-two n",
            "value": round(v, 2), "unit": "GB/s", "higher_is_better": True, "per_size": out,
            "frac_of_hbm": round(v / peak, 4), "peak": peak, "peak_kind": kind, "dtype": "f64",
            "plan_flag": args.flag,
            "config": {"workload": "C128, n = 2^12 .. 2^22, 1 GiB of input per size, iid N(0,1), "
                                   "forward + inverse; inputs larger than L2"}}


def form_batch(torch, cb, lib, dev, args):
    """20000 mixed lengths in [16, 2^20] (half 7-smooth, half with a prime
    factor <= 65537), one graph launch (one work-queue kernel) per
    execution; against the grouped schedule and against the same transforms
    as per-request plan executions."""
    import importlib
    w = importlib.import_module("catabra_b200.workloads")
    lengths = [int(v) for v in w.batch_lengths(args.count, seed=1)]
    st = torch.cuda.current_stream(dev)
    res = {}
    def timed(b, x, y):
        for _ in range(max(3, args.warmup)):
            b.execute(x, out=y)
        steps = max(3, min(args.steps, 10))
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(steps):
            b.execute(x, out=y)
        z.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(z) / steps

    for name, dt, tdt, e in (("c64", np.complex64, torch.complex64, 8),
                             ("c128", np.complex128, torch.complex128, 16)):
        t0 = time.perf_counter()
        b = cb.Batch(lengths, dt)
        t_plan = time.perf_counter() - t0
        x = torch.randn(b.total, dtype=tdt, device=dev)
        y = torch.empty_like(x)
        ms = timed(b, x, y)
        assert lib.cfft_device_faults(1) == 0
        # the grouped schedule on the same stream (context)
        bg = cb.Batch(lengths, dt, cb.BATCH_GROUPED)
        ms_g = timed(bg, x, torch.empty_like(x))
        launches_g = bg.launches()
        bg.close()
        torch.cuda.empty_cache()
        # per-request path: every transform launched on its own through its
        # cached plan (the serving engine's direct mode: one plan per length,
        # one shared two-pass scratch), host-timed from the first launch to
        # the last completion
        srv = cb.Server(dt, mode=cb.SERVE_DIRECT, max_requests=2 * len(lengths) + 16)
        srv.prepare(sorted(set(lengths)))
        xp, yp = x.data_ptr(), y.data_ptr()

        def per_request():
            for o, n in zip(b.offsets, lengths):
                srv.submit_ptr(n, xp + int(o) * e, yp + int(o) * e)
            srv.drain()
        per_request()
        t1 = time.perf_counter()
        per_request()
        ms_req = (time.perf_counter() - t1) * 1e3
        srv.close()
        nbytes = 2 * b.total * e
        res[name] = {"ms_per_batch": round(ms, 3), "GB_s": round(nbytes / (ms * 1e-3) / 1e9, 2),
                     "per_request_ms": round(ms_req, 3),
                     "per_request_GB_s": round(nbytes / (ms_req * 1e-3) / 1e9, 2),
                     "speedup_vs_per_request": round(ms_req / ms, 2), "launches": b.launches(),
                     "grouped_ms_per_batch": round(ms_g, 3), "grouped_launches": launches_g,
                     "plan_s": round(t_plan, 2), "elements": b.total}
        b.close()
        del x, y
        torch.cuda.empty_cache()
    return {"form": "batch", "metric": "FFT GB/s, one queue launch over mixed lengths",
            "value": res["c64"]["GB_s"], "unit": "GB/s", "higher_is_better": True, "per_dtype": res,
            "config": {"workload": f"{args.count} lengths log-uniform in [16, 2^20], half 7-smooth, "
                                   "half with a prime factor <= 65537 (seed 1), forward"}}


def form_serve(torch, cb, lib, dev, args):
    """Poisson arrivals at 50k req/s, n log-uniform in [64, 2^22] (80 % 7-smooth,
    20 % with a prime factor <= 65537), ComplexF32, admission cap 64 GB.
    The batched server (continuous batching) against per-request launches;
    latency = completion - submission, both on the host's steady clock."""
    import importlib
    w = importlib.import_module("catabra_b200.workloads")
    rate = 50000.0
    reqs = w.request_stream(args.count, rate, seed=1)
    lengths = [int(n) for _, n in reqs]
    e = 8
    # inputs and outputs cycle through two 8 GiB regions (far beyond L2), so
    # requests in flight together read and write distinct memory
    ring = (8 << 30) // e
    xin = torch.randn(ring, dtype=torch.complex64, device=dev)
    yout = torch.empty(ring, dtype=torch.complex64, device=dev)
    offs, cur = [], 0
    for n in lengths:
        if cur + n > ring:
            cur = 0
        offs.append(cur)
        cur += n
    def run(mode, scale):
        """Serve the stream with arrival times stretched by `scale`."""
        srv = cb.Server(np.complex64, mode=mode, max_inflight_bytes=64 << 30, max_requests=args.count + 256)
        t0 = time.perf_counter()
        distinct = sorted(set(lengths))
        srv.prepare(distinct)
        t_prep = time.perf_counter() - t0
        for n in distinct[:: max(1, len(distinct) // 64)]:     # warm the kernel variants
            srv.wait(srv.submit_ptr(n, xin.data_ptr(), yout.data_ptr()))
        torch.cuda.synchronize()
        base = srv.stats()
        xp, yp = xin.data_ptr(), yout.data_ptr()
        tickets = []
        start = time.perf_counter()
        for (ta, n), o in zip(reqs, offs):
            while time.perf_counter() - start < ta * scale:
                pass
            tickets.append(srv.submit_ptr(n, xp + o * e, yp + o * e))
        t_sub_end = time.perf_counter() - start
        srv.drain()
        wall = time.perf_counter() - start
        lat_ms = [srv.query(t) / 1e3 for t in tickets]
        st = srv.stats()
        srv.close()
        nbytes = 2 * e * sum(lengths)
        return {"p50_ms": round(_pct(lat_ms, 0.5), 3), "p99_ms": round(_pct(lat_ms, 0.99), 3),
                "mean_ms": round(statistics.mean(lat_ms), 3),
                "req_per_s": round(len(lengths) / wall, 1), "GB_s": round(nbytes / wall / 1e9, 2),
                "wall_s": round(wall, 3), "submit_s": round(t_sub_end, 3),
                "batches": st["batches"] - base["batches"],
                "launches": st["launches"] - base["launches"], "prepare_s": round(t_prep, 1)}

    res = {"batched": run(cb.SERVE_BATCHED, 1.0), "per_request": run(cb.SERVE_DIRECT, 1.0)}
    # the same stream at half the rate (25k req/s), below the batched
    # server's capacity: latency without a growing queue
    half = {"batched": run(cb.SERVE_BATCHED, 2.0), "per_request": run(cb.SERVE_DIRECT, 2.0)}
    del xin, yout
    torch.cuda.empty_cache()
    b, d = res["batched"], res["per_request"]
    return {"form": "serve", "metric": "p50/p99 latency and req/s under Poisson arrivals",
            "value": b["p99_ms"], "unit": "ms (p99, batched)", "higher_is_better": False,
            "modes": res, "speedup_req_per_s": round(b["req_per_s"] / d["req_per_s"], 2),
            "at_25k_req_per_s": half,
            "dtype": "f32",
            "config": {"workload": f"{args.count} requests, Poisson {rate:.0f} req/s (seed 1), n log-uniform "
                                   "in [64, 2^22], 80% 7-smooth / 20% prime-containing, C64, forward, "
                                   "admission cap 64 GiB, plans prepared before traffic"}}


def run_form(args):
    env = _setup_single()
    if env is None:
        return 0
    torch, cb, lib, dev = env
    fn = {"small": form_small, "precision": form_precision, "pow2": form_pow2, "batch": form_batch,
          "serve": form_serve}[args.form]
    line = fn(torch, cb, lib, dev, args)
    line.update({"n_gpus": 1, "warmup": args.warmup, "data": "synthetic (seeded)"})
    print(json.dumps(line))
    return 0


def other_forms(torch, cb, lib, dev, args):
    """The rest of the metric (plain vs batched / served, p50/p99 at the
    stated error), measured after the contract line's timed region and
    attached to it: the power-of-two sweep, the precision form, the batching
    and serving forms at their configured sizes, and the small-transform
    latency.  Each summary is the form's own line (python bench.py --form X)
    without its run bookkeeping; a form that fails records its error."""
    import copy
    out = {}
    for name, fn in (("pow2", form_pow2), ("precision", form_precision), ("batch", form_batch),
                     ("serve", form_serve), ("small", form_small)):
        a = copy.copy(args)
        a.batch, a.exps, a.flag, a.count = 0, "", "none", 20000
        a.steps = min(args.steps, 20)
        t0 = time.perf_counter()
        try:
            r = fn(torch, cb, lib, dev, a)
            for k in ("form", "n_gpus", "warmup", "data"):
                r.pop(k, None)
        except Exception as exc:                  # recorded, not fatal to the contract line
            r = {"error": f"{type(exc).__name__}: {exc}"}
        r["wall_s"] = round(time.perf_counter() - t0, 1)
        out[name] = r
        torch.cuda.empty_cache()
        cb.empty_cache()
    return out


def measure_library(torch, bufs, stream, steps=20):
    """Run-only comparison: torch.fft (cuFFT) on the same resident batches,
    fwd + inv per step.  Not the product; reported for context."""
    per = {}
    total = 0.0
    for (x, y, z), (n, b) in zip(bufs, SIZES):
        for _ in range(3):
            torch.fft.ifft(torch.fft.fft(x, dim=1), dim=1)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(steps):
            torch.fft.ifft(torch.fft.fft(x, dim=1), dim=1)
        e.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / steps
        per[str(n)] = round(ms / 2, 4)
        total += ms
    return {"value": round(algorithmic_bytes_per_step() / (total * 1e-3) / 1e9, 3), "unit": "GB/s",
            "ms_per_step": round(total, 4), "ms_per_launch": per,
            "impl": "torch.fft (cuFFT), same batches, fwd + inv"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--only", type=int, default=0, help="restrict to one transform length")
    ap.add_argument("--batch", type=int, default=0, help="override the batch (profiling cases)")
    ap.add_argument("--quick", action="store_true", help="skip the e2e and CPU-baseline legs")
    ap.add_argument("--form", default="plain", choices=FORMS,
                    help="plain (the contract line) or one of the other workload forms")
    ap.add_argument("--count", type=int, default=20000, help="batch/serve form: transforms")
    ap.add_argument("--exps", default="", help="pow2 form: comma-separated log2 lengths (default 12..22)")
    ap.add_argument("--flag", default="none", choices=("none", "measure"), help="pow2 form: plan flag")
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="reference arm: CPU seconds spread over its warm-up and timed steps")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain form: skip the other forms' summaries appended to the line")
    args = ap.parse_args()
    global SIZES
    if args.only:
        SIZES = [(n, b) for n, b in SIZES if n == args.only] or [(args.only, 1024)]
    if args.batch:
        SIZES = [(n, args.batch) for n, _ in SIZES]
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(3, args.warmup)
    if args.form != "plain":
        return run_form(args)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    cb = load_package()
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
        ms = max_over_ranks(torch, ms, dev)
    ms_step = ms / args.steps
    value = job_gbs(world, algorithmic_bytes_per_step(), ms_step)

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
    traffic = load_traffic().get(f"c128_n{n_dom}_b{b_dom}")

    e2e = None if args.quick else measure_e2e(torch, cb, lib, plans, bufs, args, world, dev)
    cufft = None if args.quick else measure_library(torch, bufs, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.quick:
        threads = os.cpu_count() or 1
        res = cpu_reference(threads, args.cpu_budget, steps=1)[0]
        cpu = {"value": round(res[0], 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"{res[2]} units (fwd+inv of one 30240 and one 10007 transform) in "
                         f"{res[1]:.1f} s, OpenMP over {threads} threads"}

    descs = []
    for h in plans:
        d = ctypes.create_string_buffer(256)
        lib.cfft_plan_describe(h, d, 256)
        descs.append(d.value.decode())
        lib.cfft_plan_destroy(h)
    dom_desc = descs[[n for n, _ in SIZES].index(n_dom)]
    forms = None
    if rank == 0 and world == 1 and not args.quick and not args.no_forms:
        del bufs
        torch.cuda.empty_cache()
        cb.empty_cache()
        forms = other_forms(torch, cb, lib, dev, args)
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
                         "kernel": f"n={n_dom} batch={b_dom}: {dom_desc}",
                         "ms_per_launch": round(ms_launch, 4)},
            "per_size_ms_per_launch": {str(n): round(m, 4) for n, _, m, _ in per},
            "plans": {str(n): d for (n, _), d in zip(SIZES, descs)},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
            "library_comparison": cufft,
            "clocks": clk.summary(),
        }
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
