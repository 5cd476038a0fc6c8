"""GPU tests of the real-input transforms (rfft / irfft / brfft).

numpy's pocketfft is the check (FFTW stand-in, as in the reference's own
tests); tolerances: 1e-12 relative L2 for float64, 1e-5 for float32.
Even n uses the half-length complex transform, odd n the complex path.
"""
import numpy as np
import pytest

from _pkg import load

pytestmark = pytest.mark.gpu

SIZES = [2, 8, 30, 4096, 30240, 10007 * 2, 65536, 3 * (1 << 18), 1, 7, 89, 10007, 30241]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available()
    return load()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_rfft_matches_numpy(cb, n, dtype):
    rng = np.random.default_rng(n)
    batch = 3
    x = rng.standard_normal((batch, n)).astype(dtype)
    tol = 1e-12 if dtype == np.float64 else 1e-5
    X = cb.rfft(x)
    assert X.shape == (batch, n // 2 + 1)
    ref = np.fft.rfft(x.astype(np.float64), axis=1)
    assert rel(X, ref) < tol
    # irfft / brfft of an arbitrary spectrum (imaginary DC/Nyquist ignored)
    S = (rng.standard_normal((batch, n // 2 + 1)) + 1j * rng.standard_normal((batch, n // 2 + 1)))
    S = S.astype(np.complex128 if dtype == np.float64 else np.complex64)
    y = cb.irfft(S, n)
    assert y.shape == (batch, n) and y.dtype == dtype
    assert rel(y, np.fft.irfft(S.astype(np.complex128), n, axis=1)) < tol
    assert rel(cb.brfft(S, n), n * np.fft.irfft(S.astype(np.complex128), n, axis=1)) < tol
    # round trip: two transforms, each within tol
    assert rel(cb.irfft(X, n), x.astype(np.float64)) < 2 * tol


def test_rfft_device_tensors_and_plans(cb):
    import torch
    n = 30240
    x = torch.randn(4, n, dtype=torch.float64, device="cuda")
    X = cb.rfft(x)
    assert X.is_cuda and X.dtype == torch.complex128 and X.shape == (4, n // 2 + 1)
    ref = np.fft.rfft(x.cpu().numpy(), axis=1)
    assert rel(X.cpu().numpy(), ref) < 1e-12
    Xc = X.clone()
    y = cb.irfft(X, n)
    assert torch.equal(X, Xc)                      # the spectrum is not modified
    assert rel(y.cpu().numpy(), x.cpu().numpy()) < 1e-12
    p = cb.plan_rfft(x.cpu().numpy(), cb.MEASURE)
    assert rel(p * x.cpu().numpy(), ref) < 1e-12
    pb = cb.plan_brfft(ref, n)
    assert rel(pb * ref, n * x.cpu().numpy()) < 1e-12


def test_rfft_invalid_direction(cb):
    import ctypes
    lib = cb._lib.LIB
    h = ctypes.c_void_p()
    cb.check(lib.cfft_rfft_plan_create(ctypes.byref(h), 64, 1, cb.C128, 0))
    buf = ctypes.c_void_p(1 << 20)
    assert lib.cfft_rfft_execute_inverse(h, buf, buf, cb.FORWARD, None) == cb._lib.ERR_INVALID
    lib.cfft_rfft_plan_destroy(h)


def test_plan_inverse_bfft_adjoint(cb):
    rng = np.random.default_rng(11)
    x = rng.standard_normal((2, 30240)) + 1j * rng.standard_normal((2, 30240))
    p = cb.plan_fft(x)
    X = p * x
    assert rel(X, np.fft.fft(x, axis=1)) < 1e-12
    assert rel(cb.plan_inv(p) * X, x) < 2e-12
    assert cb.plan_inv(p) is cb.plan_inv(p)
    pb = cb.plan_bfft(x)
    assert rel(pb * X, 30240 * x) < 2e-12
    assert rel(cb.plan_inv(pb) * (30240 * x), X) < 2e-12
    pi = cb.plan_ifft(x)
    assert rel(pi * X, x) < 2e-12
    # adjoints: <p x, y> = <x, p' y>
    y = rng.standard_normal((2, 30240)) + 1j * rng.standard_normal((2, 30240))
    for q in (p, pb, pi):
        lhs = np.vdot(q * x, y)
        rhs = np.vdot(x, q.adjoint() * y)
        assert abs(lhs - rhs) / abs(lhs) < 1e-11


def test_complex_f16(cb):
    """ComplexF16 data (the reference's self-test type), FP32 arithmetic."""
    import ctypes
    import torch
    import oracle
    n, batch = 4096, 3
    x32 = torch.randn(batch, n, dtype=torch.complex64, device="cuda")
    xh = x32.to(torch.complex32)
    y = cb.fft(xh)
    assert y.dtype == torch.complex32
    ref = oracle.fft(xh.to(torch.complex128).cpu().numpy())
    assert rel(y.to(torch.complex128).cpu().numpy(), ref) < 2e-3
    # host entry: interleaved float16 pairs
    lib = cb._lib.LIB
    h = ctypes.c_void_p()
    cb.check(lib.cfft_plan_create(ctypes.byref(h), n, batch, cb.C32, 0))
    hin = xh.cpu().view(torch.float16).numpy().copy()
    hout = np.empty_like(hin)
    cb.check(lib.cfft_execute_host(h, hin.ctypes.data_as(ctypes.c_void_p), hout.ctypes.data_as(ctypes.c_void_p), 1))
    back = hout.astype(np.float64).reshape(batch, n, 2)
    back = back[..., 0] + 1j * back[..., 1]
    ref_i = oracle.ifft(xh.to(torch.complex128).cpu().numpy())
    assert rel(back, ref_i) < 2e-3
    lib.cfft_plan_destroy(h)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_axes_and_multidim(cb, dtype):
    """Strided plans (the reference's ignored `region`): transforms along any
    axis of device tensors, fft2/fftn; host arrays through host transposes."""
    import torch
    rng = np.random.default_rng(21)
    x = (rng.standard_normal((6, 30240 // 6 // 7, 7 * 6)) + 1j * rng.standard_normal((6, 720, 42))).astype(dtype)
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    xd = torch.from_numpy(x).cuda()
    for axis in (0, 1, 2, -1):
        ref = np.fft.fft(x.astype(np.complex128), axis=axis)
        assert rel(cb.fft(xd, axis=axis).cpu().numpy(), ref) < tol, axis
        assert rel(cb.fft(x, axis=axis), ref) < tol, axis
    ref2 = np.fft.fft2(x.astype(np.complex128))
    assert rel(cb.fft2(xd).cpu().numpy(), ref2) < 2 * tol
    refn = np.fft.fftn(x.astype(np.complex128))
    assert rel(cb.fftn(xd).cpu().numpy(), refn) < 3 * tol
    assert rel(cb.ifftn(cb.fftn(xd)).cpu().numpy(), x) < 6 * tol


def test_plan_many_strided_abi(cb):
    """cfft_plan_create_many through the C ABI: the second axis of a
    column-major n1 x n2 matrix (stride n1, distance 1)."""
    import ctypes
    import torch
    n1, n2 = 96, 1000
    rng = np.random.default_rng(5)
    A = rng.standard_normal((n2, n1)) + 1j * rng.standard_normal((n2, n1))   # row-major view of column-major n1 x n2
    d = torch.from_numpy(A).cuda()
    y = torch.empty_like(d)
    lib = cb._lib.LIB
    h = ctypes.c_void_p()
    cb.check(lib.cfft_plan_create_many(ctypes.byref(h), n2, n1, cb.C128, 0, n1, 1, n1, 1))
    cb.check(lib.cfft_execute(h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(y.data_ptr()), 0,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    assert rel(y.cpu().numpy(), np.fft.fft(A, axis=0)) < 1e-12
    lib.cfft_plan_destroy(h)
