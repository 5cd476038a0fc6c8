"""GPU parity at the configured sizes: the benchmarked batches, two-pass plans
whose batch spans several scratch chunks, and the persistent n = 4096 kernel
with more transforms than it has CTAs.  Sampled rows are compared with the
oracle (the CPU restatement of CatabraFFT.jl's algorithm).

Bars (relative L2): 1e-12 for ComplexF64 against the oracle, 1e-5 for
ComplexF32 against the FP64 oracle.  Where the reference algorithm itself
drifts from the exact DFT by more than that (its twiddle recurrences at large
primes), the GPU result must be within 1e-12 of the exact DFT and within the
oracle's own distance to it (plus 1e-12) of the oracle.
"""
import ctypes

import numpy as np
import pytest

import oracle
from _pkg import load

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available()
    return load()


def _device_batch(torch, n, batch, dtype, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    real = torch.float64 if dtype == np.complex128 else torch.float32
    return torch.complex(torch.randn(batch, n, dtype=real, device="cuda", generator=g),
                         torch.randn(batch, n, dtype=real, device="cuda", generator=g))


def _execute(cb, plan, x, direction, out=None):
    import torch
    y = torch.empty_like(x) if out is None else out
    stream = torch.cuda.current_stream().cuda_stream
    cb.check(cb._lib.LIB.cfft_execute(plan, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                      direction, ctypes.c_void_p(stream)))
    return y


class _CPlan:
    """A plan made through the C ABI (cfft_plan_create), released on exit."""

    def __init__(self, cb, n, batch, dtype_code, flags=0):
        self.cb = cb
        self.h = ctypes.c_void_p()
        cb.check(cb._lib.LIB.cfft_plan_create(ctypes.byref(self.h), n, batch, dtype_code, flags))

    def describe(self):
        buf = ctypes.create_string_buffer(512)
        self.cb.check(self.cb._lib.LIB.cfft_plan_describe(self.h, buf, 512))
        return buf.value.decode()

    def launches(self):
        return self.cb._lib.LIB.cfft_plan_launches(self.h)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.cb._lib.LIB.cfft_plan_destroy(self.h)


def _bar(ref, x):
    """1e-12, or the oracle's own distance to the exact DFT plus 1e-12."""
    return max(TOL64, rel(ref, np.fft.fft(x)) + TOL64)


@pytest.mark.parametrize("n", [30240, 10007])
def test_bench_configuration_rows_vs_oracle(cb, n):
    """The benchmarked configuration itself: 1024 transforms of n = 30240
    (mixed radix) or n = 10007 (Rader), forward and inverse, rows 0, 511 and
    1023 against the oracle; the plans are the benchmark's: a cluster of
    nine register 3360-point CTAs (input by tensor copies) for 30240, a
    cluster of five register 4096-point CTAs for 10007's convolution."""
    import torch
    batch = 1024
    x = _device_batch(torch, n, batch, np.complex128, seed=n)
    with _CPlan(cb, n, batch, cb.C128) as p:
        desc = p.describe()
        assert ("cluster(C=9,L=3360 per CTA,threads=240,tma)" in desc) == (n == 30240), desc
        assert ("rader(n=10007,M=20480)+cluster(C=5" in desc) == (n == 10007), desc
        y = _execute(cb, p.h, x, cb.FORWARD)
        z = _execute(cb, p.h, x, cb.INVERSE)
        torch.cuda.synchronize()
    rows = [0, 511, 1023]
    xs = x[rows].cpu().numpy()
    ys, zs = y[rows].cpu().numpy(), z[rows].cpu().numpy()
    for i, r in enumerate(rows):
        assert rel(ys[i], oracle.fft(xs[i])) < TOL64, (n, r, "fft")
        assert rel(zs[i], oracle.ifft(xs[i])) < TOL64, (n, r, "ifft")


@pytest.mark.parametrize("n,batch,dtype", [(3 ** 10, 300, np.complex64), (3 ** 12, 9, np.complex128),
                                           (999983, 3, np.complex128)])
def test_two_pass_across_scratch_chunks(cb, n, batch, dtype):
    """Generic two-pass plans whose batch is processed in several scratch
    chunks (the intermediate of one chunk is sized to stay in L2):
    ComplexF32 3^10 x 300, ComplexF64 3^12 x 9, and the prime 999983, whose
    convolution exceeds a cluster and runs as a two-pass Bluestein plan, one
    transform per chunk.  (Power-of-two chunking is covered below.)"""
    import torch
    code = cb.C128 if dtype == np.complex128 else cb.C64
    x = _device_batch(torch, n, batch, dtype, seed=n + batch)
    with _CPlan(cb, n, batch, code) as p:
        desc = p.describe()
        assert "twopass" in desc, desc
        stages = 2 if "bluestein" not in desc else 4
        assert p.launches() > stages, (desc, p.launches())     # more than one chunk ran
        y = _execute(cb, p.h, x, cb.FORWARD)
        z = _execute(cb, p.h, x, cb.INVERSE)
        torch.cuda.synchronize()
    rows = sorted({0, batch // 2, batch - 1})
    xs = x[rows].cpu().numpy().astype(np.complex128)
    ys, zs = y[rows].cpu().numpy(), z[rows].cpu().numpy()
    for i, r in enumerate(rows):
        ref, iref = oracle.fft(xs[i]), oracle.ifft(xs[i])
        if dtype == np.complex64:
            assert rel(ys[i], ref) < TOL32, (n, r)
            assert rel(zs[i], iref) < TOL32, (n, r)
        else:
            bar = _bar(ref, xs[i])
            assert rel(ys[i], ref) < bar, (n, r, bar)
            assert rel(ys[i], np.fft.fft(xs[i])) < TOL64, (n, r)
            assert rel(zs[i], iref) < bar, (n, r)


@pytest.mark.parametrize("dtype,tol", [(np.complex128, TOL64), (np.complex64, TOL32)])
def test_register_kernel_persistent_loop(cb, dtype, tol):
    """n = 4096 on persistent CTAs (as many as are co-resident, about three per
    SM): with 1000 and 2000 transforms every CTA runs several iterations, so
    the prefetch of its next transform into the freed shared buffer is
    exercised.  Every row forward, inverse and backward against the oracle,
    and in place."""
    import torch
    n = 4096
    code = cb.C128 if dtype == np.complex128 else cb.C64
    for batch in (1000, 2000):
        x = _device_batch(torch, n, batch, dtype, seed=batch)
        xs = x.cpu().numpy().astype(np.complex128)
        with _CPlan(cb, n, batch, code) as p:
            assert "+r4096" in p.describe(), p.describe()
            outs = [_execute(cb, p.h, x, d) for d in (cb.FORWARD, cb.INVERSE, cb.BACKWARD)]
            t = x.clone()
            _execute(cb, p.h, t, cb.FORWARD, out=t)               # in place
            torch.cuda.synchronize()
        refs = [oracle.transform(xs, d) for d in (oracle.FWD, oracle.INV, oracle.BWD)]
        for d, (o, r) in enumerate(zip(outs, refs)):
            o = o.cpu().numpy()
            errs = np.linalg.norm(o - r, axis=1) / np.linalg.norm(r, axis=1)
            assert errs.max() < tol, (batch, d, int(errs.argmax()), float(errs.max()))
        assert np.array_equal(t.cpu().numpy(), outs[0].cpu().numpy())


def _greedy_split(L):
    out = []
    while L > 1:
        r = next(r for r in (16, 9, 8, 7, 5, 4, 3, 2) if L % r == 0)
        out.append(r)
        L //= r
    return out


def _pow2_check(cb, n, batch, dtype, desc_part, flags=0):
    import torch
    code = cb.C128 if dtype == np.complex128 else cb.C64
    tol = TOL64 if dtype == np.complex128 else TOL32
    x = _device_batch(torch, n, batch, dtype, seed=n + batch)
    with _CPlan(cb, n, batch, code, flags) as p:
        assert desc_part in p.describe(), (n, p.describe())
        outs = [_execute(cb, p.h, x, d) for d in (cb.FORWARD, cb.INVERSE, cb.BACKWARD)]
        t = x.clone()
        _execute(cb, p.h, t, cb.FORWARD, out=t)                   # in place
        torch.cuda.synchronize()
    rows = sorted({0, batch // 2, batch - 1})
    xs = x[rows].cpu().numpy().astype(np.complex128)
    for d, o in zip((oracle.FWD, oracle.INV, oracle.BWD), outs):
        ref = oracle.transform(xs, d)
        got = o[rows].cpu().numpy()
        errs = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert errs.max() < tol, (n, batch, d, float(errs.max()))
    assert np.array_equal(t[rows].cpu().numpy(), outs[0][rows].cpu().numpy())


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_pow2_register_passes(cb, dtype):
    """Power-of-two n = N1 x 4096 (N1 = 2 .. 1024): up to 2^16 one pass on a
    cluster of N1 register 4096-point CTAs; beyond, pass A (the n = 4096
    kernel over the stride-N1 subsequences; ComplexF64 loads them by tensor
    copies) and pass B (the N1-point column DFTs).  Batches give every
    persistent CTA several rows and tiles (prefetch into the freed buffer),
    and the largest lengths run several intermediate chunks.  ComplexF32
    takes pass A by tensor copies of subsequence pairs.  Forward,
    inverse, backward and in place against the oracle; no kernel recorded a
    timed-out wait."""
    cb._lib.LIB.cfft_device_faults(1)
    for e in range(13, 23):
        n = 1 << e
        N1 = n // 4096
        batch = max(3, 2048 // N1 + 1)
        if n <= 16384:                              # one pass on a cluster of N1 CTAs
            _pow2_check(cb, n, batch, dtype, f"pow2cluster(C={N1},4096 per CTA,ctas_per_sm=2)")
        else:
            shape = "ctas_per_sm=2,tma)"
            _pow2_check(cb, n, batch, dtype, f"pow2(N1={N1},N2=4096,{shape}")
    assert cb._lib.LIB.cfft_device_faults(1) == 0


def test_pow2_other_variants(cb, tmp_path):
    """Every ComplexF64 build of pass A, reached through wisdom entries for
    MEASURE plans: cp.async loads and tensor copies, at three and at two CTAs
    per SM."""
    variants = [(3, 0, ")"), (2, 0, ")"), (3, 1, ",tma)"), (2, 1, ",tma)")]
    cases = [(1 << 13, 300), (1 << 14, 150), (1 << 15, 80), (1 << 16, 40), (1 << 20, 3), (1 << 22, 9)]
    cb._lib.LIB.cfft_device_faults(1)
    for mb, var, tag in variants:
        lines = ["catabra-b200-wisdom 1"]
        for n, batch in cases:
            N1 = n // 4096
            sig = f"4 0 {n} {N1} 4096 1 {mb} a {' '.join(map(str, _greedy_split(N1)))} c 16 16 16"
            if var:
                sig += f" v{var}"
            lines.append(f"{n} {batch} 0 {cb.MEASURE} | {sig}")
        path = tmp_path / f"w{mb}{var}.txt"
        path.write_text("\n".join(lines) + "\n")
        cb.forget_wisdom()
        cb.import_wisdom(str(path))
        try:
            for n, batch in cases:
                _pow2_check(cb, n, batch, np.complex128, f"pow2(N1={n // 4096},N2=4096,ctas_per_sm={mb}{tag}",
                            flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()
    assert cb._lib.LIB.cfft_device_faults(1) == 0


def test_pow2_c64_pass_a_variants(cb, tmp_path):
    """Both ComplexF32 builds of pass A through wisdom entries for MEASURE
    plans: per-element cp.async at three CTAs per SM, and tensor copies of
    subsequence pairs at two (64 KB pair buffer; N1 = 2 is a single pair per
    transform), against the oracle at 1e-5."""
    variants = [(3, 0, ")"), (2, 1, ",tma)")]
    cases = [(1 << 13, 120), (1 << 15, 40), (1 << 16, 21), (1 << 20, 3), (1 << 22, 2)]
    cb._lib.LIB.cfft_device_faults(1)
    for mb, var, tag in variants:
        lines = ["catabra-b200-wisdom 1"]
        for n, batch in cases:
            N1 = n // 4096
            sig = f"4 0 {n} {N1} 4096 1 {mb} a {' '.join(map(str, _greedy_split(N1)))} c 16 16 16"
            if var:
                sig += f" v{var}"
            lines.append(f"{n} {batch} {cb.C64} {cb.MEASURE} | {sig}")
        path = tmp_path / f"c64w{mb}{var}.txt"
        path.write_text("\n".join(lines) + "\n")
        cb.forget_wisdom()
        cb.import_wisdom(str(path))
        try:
            for n, batch in cases:
                _pow2_check(cb, n, batch, np.complex64, f"pow2(N1={n // 4096},N2=4096,ctas_per_sm={mb}{tag}",
                            flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()
    assert cb._lib.LIB.cfft_device_faults(1) == 0


def test_pow2_cluster_three_ctas_per_sm(cb, tmp_path):
    """The single-pass cluster kernels not chosen by default, reached through
    wisdom entries for MEASURE plans, both element types: three CTAs per SM
    for every C, and two CTAs per SM for the 8- and 16-CTA clusters."""
    cases = [(1 << 13, 300, 3), (1 << 14, 150, 3), (1 << 15, 80, 3), (1 << 16, 40, 3), (1 << 15, 80, 2),
             (1 << 16, 40, 2)]
    for dtype, code in ((np.complex128, 0), (np.complex64, 1)):
        lines = ["catabra-b200-wisdom 1"]
        for n, batch, mb in cases[:4]:
            C = n // 4096
            lines.append(f"{n} {batch} {code} {cb.MEASURE} | 8 0 {n} {C} 4096 {C} {mb} a c 16 16 16")
        path = tmp_path / f"c{code}.txt"
        path.write_text("\n".join(lines) + "\n")
        cb.forget_wisdom()
        cb.import_wisdom(str(path))
        try:
            for n, batch, mb in cases[:4]:
                _pow2_check(cb, n, batch, dtype, f"pow2cluster(C={n // 4096},4096 per CTA,ctas_per_sm={mb})",
                            flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()
        lines = ["catabra-b200-wisdom 1"]
        for n, batch, mb in cases[4:]:
            C = n // 4096
            lines.append(f"{n} {batch} {code} {cb.MEASURE} | 8 0 {n} {C} 4096 {C} {mb} a c 16 16 16")
        path.write_text("\n".join(lines) + "\n")
        cb.import_wisdom(str(path))
        try:
            for n, batch, mb in cases[4:]:
                _pow2_check(cb, n, batch, dtype, f"pow2cluster(C={n // 4096},4096 per CTA,ctas_per_sm={mb})",
                            flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()


def test_pow2_dataflow_single_launch(cb, tmp_path):
    """Both power-of-two passes in one persistent dataflow launch (rows and
    column tiles claimed from a ticket, per-transform counters, a ring of
    intermediates), reached through wisdom entries for MEASURE plans: one
    launch per execution, every variant's parity, no timed-out wait."""
    cases = [(1 << 15, 600), (1 << 16, 300), (1 << 18, 40), (1 << 20, 9), (1 << 22, 5)]
    cb._lib.LIB.cfft_device_faults(1)
    for dtype, code in ((np.complex128, 0), (np.complex64, 1)):
        lines = ["catabra-b200-wisdom 1"]
        for n, batch in cases:
            N1 = n // 4096
            sig = f"4 0 {n} {N1} 4096 1 2 a {' '.join(map(str, _greedy_split(N1)))} c 16 16 16 v2"
            lines.append(f"{n} {batch} {code} {cb.MEASURE} | {sig}")
        path = tmp_path / f"f{code}.txt"
        path.write_text("\n".join(lines) + "\n")
        cb.forget_wisdom()
        cb.import_wisdom(str(path))
        try:
            for n, batch in cases:
                with _CPlan(cb, n, batch, cb.C128 if code == 0 else cb.C64, cb.MEASURE) as p:
                    assert p.launches() == 1, (n, p.describe())
                _pow2_check(cb, n, batch, dtype, f"pow2(N1={n // 4096},N2=4096,ctas_per_sm=2,dataflow)",
                            flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()
    assert cb._lib.LIB.cfft_device_faults(1) == 0


def test_mixed_cluster_tensor_copy_variants(cb, tmp_path):
    """The ComplexF64 mixed-radix cluster kernels that load each CTA's
    stride-C subsequence by tensor copies (30240 as 7 x 4320 and as
    9 x 3360), reached through wisdom entries for MEASURE plans: forward,
    inverse, backward and in place against the oracle, with a batch that
    gives several transforms per cluster slot; no copy timed out."""
    cb._lib.LIB.cfft_device_faults(1)
    for sig, tag in (("7 0 30240 7 4320 7 288 a c v4", "cluster(C=7,L=4320 per CTA,threads=288,tma)"),
                     ("7 0 30240 9 3360 9 240 a c v5", "cluster(C=9,L=3360 per CTA,threads=240,tma)")):
        path = tmp_path / "mix.txt"
        path.write_text(f"catabra-b200-wisdom 1\n30240 70 {cb.C128} {cb.MEASURE} | {sig}\n")
        cb.forget_wisdom()
        cb.import_wisdom(str(path))
        try:
            _pow2_check(cb, 30240, 70, np.complex128, tag, flags=cb.MEASURE)
        finally:
            cb.forget_wisdom()
    assert cb._lib.LIB.cfft_device_faults(1) == 0


def test_pow2_cluster_tensor_copy_variant(cb, tmp_path):
    """The ComplexF64 single-pass cluster kernel that loads each CTA's
    stride-C subsequence by tensor copies (a timed candidate, slower than the
    direct loads at 8192 and 16384), reached through wisdom entries for
    MEASURE plans: every cluster size against the oracle, no copy timed out."""
    cases = [(1 << 13, 300), (1 << 14, 150), (1 << 15, 80), (1 << 16, 40)]
    cb._lib.LIB.cfft_device_faults(1)
    lines = ["catabra-b200-wisdom 1"]
    for n, batch in cases:
        C = n // 4096
        lines.append(f"{n} {batch} {cb.C128} {cb.MEASURE} | 8 0 {n} {C} 4096 {C} 2 a c 16 16 16 v1")
    path = tmp_path / "p2cl_tma.txt"
    path.write_text("\n".join(lines) + "\n")
    cb.forget_wisdom()
    cb.import_wisdom(str(path))
    try:
        for n, batch in cases:
            _pow2_check(cb, n, batch, np.complex128, f"pow2cluster(C={n // 4096},4096 per CTA,ctas_per_sm=2,tma)",
                        flags=cb.MEASURE)
    finally:
        cb.forget_wisdom()
    assert cb._lib.LIB.cfft_device_faults(1) == 0
