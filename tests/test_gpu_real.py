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
