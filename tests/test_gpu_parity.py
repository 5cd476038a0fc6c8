"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bars (relative L2): 1e-12 for ComplexF64 against the oracle's restatement of
the reference algorithm, 1e-5 for the ComplexF32 form against the FP64
oracle.  Where the reference algorithm itself drifts from the exact DFT (its
twiddle recurrences, see the fixtures' recorded errors), the bar is the
oracle's own distance to the exact DFT plus 1e-12.
"""
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


def cplx(rng, shape, dtype=np.complex128):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def test_golden_fixtures_c128(cb, golden128):
    for n in golden128["meta_n"]:
        n = int(n)
        x = golden128[f"x_{n}"]
        assert rel(cb.fft(x), golden128[f"fft_{n}"]) < TOL64, n
        if f"ifft_{n}" in golden128:
            assert rel(cb.ifft(x), golden128[f"ifft_{n}"]) < TOL64, n


def test_golden_fixtures_c64(cb, golden64):
    for key in golden64:
        if not key.startswith("x_"):
            continue
        n = int(key[2:])
        y = cb.fft(golden64[key])
        assert y.dtype == np.complex64
        assert rel(y, golden64[f"fft_{n}"]) < TOL32, n


@pytest.mark.parametrize("n", [10, 100, 1000, 10 ** 4, 10 ** 5, 10 ** 6])
def test_mixed_radix_sizes(cb, n):
    # runtests.jl:9-15 (10^7 is in test_largest_mixed)
    rng = np.random.default_rng(n)
    x = cplx(rng, n)
    ref = oracle.fft(x)
    ex = np.fft.fft(x)
    bar = max(TOL64, rel(ref, ex) + TOL64)
    assert rel(cb.fft(x), ref) < bar
    assert rel(cb.ifft(x), oracle.ifft(x)) < bar


def test_largest_mixed(cb):
    n = 10 ** 7
    rng = np.random.default_rng(7)
    x = cplx(rng, n)
    ref = oracle.fft(x)
    ex = np.fft.fft(x)
    got = cb.fft(x)
    assert rel(got, ex) < TOL64
    assert rel(got, ref) < rel(ref, ex) + TOL64


@pytest.mark.parametrize("n", [11, 13, 17, 19, 43, 89, 1721, 257, 5003, 10007, 65537])
def test_rader_sizes(cb, n):
    rng = np.random.default_rng(n)
    x = cplx(rng, n)
    ref = oracle.fft(x)
    bar = max(TOL64, rel(ref, np.fft.fft(x)) + TOL64) if n > 20000 else TOL64
    assert rel(cb.fft(x), ref) < bar, cb.describe_strategy(n)
    assert rel(cb.ifft(x), oracle.ifft(x)) < bar


@pytest.mark.parametrize("b,maxexp", [(2, 20), (3, 13), (5, 10), (7, 8)])
def test_pure_radix_families(cb, b, maxexp):
    rng = np.random.default_rng(b)
    for e in range(1, maxexp + 1):
        n = b ** e
        x = cplx(rng, n)
        assert rel(cb.fft(x), oracle.fft(x)) < TOL64, (n, cb.describe_strategy(n))
        assert rel(cb.ifft(x), oracle.ifft(x)) < TOL64, n


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 15, 16, 30, 64, 120])
def test_tiny_sizes_and_bfft(cb, n):
    rng = np.random.default_rng(n + 100)
    x = cplx(rng, n)
    assert rel(cb.fft(x), oracle.fft(x)) < TOL64
    assert rel(cb.bfft(x), oracle.bfft(x)) < TOL64


def test_selftest_roundtrip_f64_f32(cb):
    # runtests.jl:39-46 (ComplexF16 is not a supported element type here)
    rng = np.random.default_rng(1)
    for n in [89, 121, 2 ** 10, 2 ** 11, 3 ** 7, 5 ** 6, 10 ** 4]:
        x = cplx(rng, n)
        assert rel(cb.ifft(cb.fft(x)), x) < TOL64
        x32 = x.astype(np.complex64)
        assert rel(cb.ifft(cb.fft(x32)), x32) < TOL32


@pytest.mark.parametrize("n,batch", [(4096, 37), (30240, 6), (10007, 5), (89, 300), (17, 1000),
                                     (2 ** 20, 3), (10006, 4), (19683, 3)])
def test_batched_equals_single(cb, n, batch):
    rng = np.random.default_rng(n)
    x = cplx(rng, (batch, n))
    y = cb.fft(x)
    for b in [0, batch // 2, batch - 1]:
        assert rel(y[b], oracle.fft(x[b])) < max(TOL64, rel(oracle.fft(x[b]), np.fft.fft(x[b])) + TOL64)
    single = cb.fft(np.ascontiguousarray(x[batch - 1]))
    assert np.array_equal(single, y[batch - 1])      # same plan shape -> bitwise


@pytest.mark.parametrize("n", [2 ** 16, 3 ** 9, 30240, 10007, 4096])
def test_fp32_form_error_vs_fp64_oracle(cb, n):
    rng = np.random.default_rng(n)
    x = (rng.uniform(-1, 1, (4, n)) + 1j * rng.uniform(-1, 1, (4, n))).astype(np.complex64)
    y = cb.fft(x)
    ref = oracle.fft(x.astype(np.complex128))
    assert rel(y, ref) < TOL32, cb.describe_strategy(n, np.complex64)
    assert rel(cb.ifft(x), oracle.ifft(x.astype(np.complex128))) < TOL32


def test_device_path_matches_host_path(cb):
    import torch
    rng = np.random.default_rng(3)
    for n, batch in [(4096, 8), (30240, 2), (10007, 2)]:
        x = cplx(rng, (batch, n))
        host = cb.fft(x)
        dev = cb.fft(torch.from_numpy(x).cuda())
        torch.cuda.synchronize()
        assert np.array_equal(dev.cpu().numpy(), host)


def test_inplace_and_input_untouched(cb):
    import torch
    rng = np.random.default_rng(4)
    for n in [4096, 30240, 10007, 2 ** 20]:
        x = cplx(rng, n)
        keep = x.copy()
        y = cb.fft(x)
        assert np.array_equal(x, keep)                  # input never modified
        t = torch.from_numpy(x).cuda()
        cb.fft_(t)
        torch.cuda.synchronize()
        assert rel(t.cpu().numpy(), y) < 1e-15
        z = x.copy()
        cb.fft_(z)
        assert rel(z, y) < 1e-15


def test_plan_flags_measure_enchant(cb):
    rng = np.random.default_rng(5)
    for n in [4096, 30240, 10007]:
        x = cplx(rng, (2, n))
        base = cb.fft(x)
        for flag in (cb.MEASURE, cb.ENCHANT):
            p = cb.plan_fft(x, flag)
            assert rel(p * x, base) < TOL64, (n, flag, p.describe())
            y = np.empty_like(x)
            cb.mul_(y, p, x)
            assert rel(y, base) < TOL64


def test_exact_twiddles_flag(cb):
    rng = np.random.default_rng(6)
    n = 10007
    x = cplx(rng, n)
    p = cb.plan_fft(x, cb.EXACT_TWIDDLES)
    assert rel(p * x, np.fft.fft(x)) < 1e-14      # exact W: closer to the true DFT
    assert rel(p * x, oracle.fft(x)) < TOL64


def test_full_size_properties(cb):
    # configuration sizes: linearity, Parseval, round trip (size-independent)
    import torch
    rng = np.random.default_rng(8)
    for n, batch in [(30240, 64), (10007, 64), (4096, 256)]:
        a = torch.from_numpy(cplx(rng, (batch, n))).cuda()
        b = torch.from_numpy(cplx(rng, (batch, n))).cuda()
        fa, fb = cb.fft(a), cb.fft(b)
        fab = cb.fft(2.0 * a - 3.0 * b)
        assert (torch.linalg.norm(fab - (2.0 * fa - 3.0 * fb)) / torch.linalg.norm(fab)).item() < 1e-13
        parse = (torch.linalg.norm(fa) ** 2 / (n * torch.linalg.norm(a) ** 2)).item()
        assert abs(parse - 1.0) < 1e-12
        back = cb.ifft(fa)
        # Rader round trip carries the reference twiddle error twice (~8e-13)
        assert (torch.linalg.norm(back - a) / torch.linalg.norm(a)).item() < TOL64


def test_empty_cache_releases_plans(cb):
    x = np.ones(4096, dtype=np.complex128)
    cb.fft(x)
    cb.empty_cache()
    assert rel(cb.fft(x)[:1], np.array([4096.0 + 0j])) < 1e-15


@pytest.mark.parametrize("dtype,tol", [(np.complex128, TOL64), (np.complex64, TOL32)])
def test_register_kernel_n4096(cb, dtype, tol):
    # n = 4096 runs the register kernel (16 x 16 x 16, one transform per CTA);
    # forward / inverse / backward against the oracle, batched and single,
    # in place, and through the descriptor-driven batch path
    import torch
    rng = np.random.default_rng(4096)
    n = 4096
    for batch in (1, 3, 300):
        x = cplx(rng, (batch, n), dtype)
        p = cb.plan_fft(x)
        assert "+r4096" in p.describe(), p.describe()
        xx = x.astype(np.complex128)
        assert rel(cb.fft(x), oracle.fft(xx)) < tol
        assert rel(cb.ifft(x), oracle.ifft(xx)) < tol
        assert rel(cb.bfft(x), oracle.bfft(xx)) < tol
    t = torch.from_numpy(x).cuda()
    y = cb.fft(x)
    cb.fft_(t)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), y)
    b = cb.Batch([n, 30240, n], dtype)
    xb = cplx(rng, b.total, dtype)
    yb = b.execute(torch.from_numpy(xb).cuda()).cpu().numpy()
    for o, m in zip(b.offsets, [n, 30240, n]):
        assert rel(yb[o:o + m], oracle.fft(xb[o:o + m].astype(np.complex128))) < tol, m
    b.close()
