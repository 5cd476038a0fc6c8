"""ComplexF16 and strided plans that read and write the caller's layout in
their own first and last kernel (KParams in_fmt / out_fmt).

The reference runs Float16 through its generic Julia path (test/runtests.jl:39)
and ignores `region` (src/CatabraFFT.jl:169).  Here a ComplexF16 or strided
plan whose stages are generic kernels is fused: it issues exactly the plain
plan's launches, and its result is bit-identical to the plain plan run on the
widened (gathered) data and narrowed (scattered) afterwards, the same
arithmetic in one sweep.  Plans on the register kernels keep their separate
widening / gathering kernels (reported as two more launches).
"""
import ctypes

import numpy as np
import pytest

import oracle
from _pkg import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available()
    return load()


def _plan(cb, n, batch, dtype):
    h = ctypes.c_void_p()
    cb.check(cb._lib.LIB.cfft_plan_create(ctypes.byref(h), n, batch, dtype, cb.NO_FLAG))
    return h


def _desc(cb, h):
    buf = ctypes.create_string_buffer(256)
    cb._lib.LIB.cfft_plan_describe(h, buf, 256)
    return buf.value.decode()


def _run(cb, h, x, y, d=0):
    import torch
    vp = ctypes.c_void_p
    cb.check(cb._lib.LIB.cfft_execute(h, vp(x.data_ptr()), vp(y.data_ptr()), d,
                                      vp(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()


# (n, fused): generic shapes fuse; the register kernels (4096, pow2, the 30240
# cluster, Rader primes up to 16385) keep their separate sweeps
F16_CASES = [(1000, True), (19683, True), (6000, True), (999983, True), (2 * 3 ** 9 * 5, True),
             (4096, False), (1 << 16, False), (30240, False), (10007, False)]


@pytest.mark.parametrize("n,fused", F16_CASES)
def test_complex_f16_fused(cb, n, fused):
    import torch
    lib = cb._lib.LIB
    batch = 3 if n > 100000 else 7
    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    x32 = torch.complex(torch.randn(batch, n, device="cuda", generator=g),
                        torch.randn(batch, n, device="cuda", generator=g))
    xh = x32.to(torch.complex32)
    hh, hf = _plan(cb, n, batch, cb.C32), _plan(cb, n, batch, cb.C64)
    desc = _desc(cb, hh)
    assert desc.startswith("f16+" if fused else "f16io+"), desc
    plain = lib.cfft_plan_launches(hf)
    assert lib.cfft_plan_launches(hh) == (plain if fused else plain + 2)
    for d in (0, 1, 2):
        yh = torch.empty_like(xh)
        _run(cb, hh, xh, yh, d)
        w = xh.to(torch.complex64)                       # exact widening
        y32 = torch.empty_like(w)
        _run(cb, hf, w, y32, d)
        expect = y32.to(torch.complex32)                 # one round-to-nearest narrowing
        assert torch.equal(yh.view(torch.float16), expect.view(torch.float16)), (n, d)
    ref = oracle.fft(xh.to(torch.complex128).cpu().numpy()[0])
    yf = torch.empty_like(xh)
    _run(cb, hh, xh, yf, 0)
    r = yf.to(torch.complex128).cpu().numpy()[0]
    assert np.linalg.norm(r - ref) / np.linalg.norm(ref) < 2e-3
    # in place
    t = xh.clone()
    _run(cb, hh, t, t, 0)
    assert torch.equal(t.view(torch.float16), yf.view(torch.float16))
    lib.cfft_plan_destroy(hh)
    lib.cfft_plan_destroy(hf)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
@pytest.mark.parametrize("n,fused", [(1000, True), (19683, True), (999983, True), (4096, False), (1 << 16, False)])
def test_strided_fused(cb, dtype, n, fused):
    """The second axis of a column-major n1 x n matrix (stride n1, distance
    1) and a padded row layout (stride 2, distance 2 n + 3)."""
    import torch
    lib = cb._lib.LIB
    code = cb.C128 if dtype == np.complex128 else cb.C64
    n1 = 5
    rng = np.random.default_rng(n)
    for stride, dist, total in ((n1, 1, n * n1), (2, 2 * n + 3, (2 * n + 3) * n1)):
        buf = (rng.standard_normal(total) + 1j * rng.standard_normal(total)).astype(dtype)
        d = torch.from_numpy(buf).cuda()
        y = torch.zeros_like(d)
        h = ctypes.c_void_p()
        cb.check(lib.cfft_plan_create_many(ctypes.byref(h), n, n1, code, 0, stride, dist, stride, dist))
        desc = _desc(cb, h)
        assert ("strided(fused)+" in desc) == fused, desc
        hp = _plan(cb, n, n1, code)
        plain = lib.cfft_plan_launches(hp)
        assert lib.cfft_plan_launches(h) == (plain if fused else plain + 2)
        _run(cb, h, d, y, 0)
        idx = np.arange(n1)[:, None] * dist + np.arange(n)[None, :] * stride
        xg = torch.from_numpy(buf[idx]).cuda()
        yg = torch.empty_like(xg)
        _run(cb, hp, xg, yg, 0)
        got = y.cpu().numpy()
        assert np.array_equal(got[idx], yg.cpu().numpy()), (n, stride)
        untouched = np.ones(total, bool)
        untouched[idx.ravel()] = False
        assert not got[untouched].any()                      # nothing written between the elements
        ref = oracle.fft(buf[idx][0].astype(np.complex128))
        tol = 1e-12 if dtype == np.complex128 else 1e-5
        if dtype == np.complex128:
            tol = max(tol, np.linalg.norm(ref - np.fft.fft(buf[idx][0])) / np.linalg.norm(ref) + 1e-12)
        assert np.linalg.norm(got[idx][0] - ref) / np.linalg.norm(ref) < tol
        # in place
        t = d.clone()
        _run(cb, h, t, t, 0)
        assert np.array_equal(t.cpu().numpy()[idx], got[idx])
        lib.cfft_plan_destroy(h)
        lib.cfft_plan_destroy(hp)
