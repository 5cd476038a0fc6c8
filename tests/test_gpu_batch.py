"""GPU tests of the batched form: one graph launch over mixed lengths.

Both schedules run: the single persistent launch over a queue of work items
(the default; the graph holds exactly one kernel) and the grouped launches
(CFFT_BATCH_GROUPED).  Every transform of a seeded mixed batch (half 7-smooth lengths, half with a
prime factor up to 65537) is compared with the oracle: 1e-12 relative L2 for
ComplexF64 (or, where the reference algorithm's own twiddle recurrences
drift further from the exact DFT, that drift plus 1e-12), and 1e-5 against
the FP64 oracle for ComplexF32.
"""
import numpy as np
import pytest

import oracle
from _pkg import load

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def bar64(ref, x):
    """1e-12, or the oracle's own distance to the exact DFT plus 1e-12."""
    return max(1e-12, rel(ref, np.fft.fft(x)) + 1e-12)


@pytest.fixture(scope="module")
def cb():
    import torch
    assert torch.cuda.is_available()
    return load()


def _lengths(cb, count, seed, hi):
    import importlib
    w = importlib.import_module("catabra_b200.workloads")
    return w.batch_lengths(count, seed=seed, lo=16, hi=hi)


SCHEDULES = [0, 32]                                # queue, CFFT_BATCH_GROUPED


def _check_launches(b, flags):
    if flags == 0:
        assert b.launches() == 1                   # one work-queue kernel
    else:
        assert b.launches() >= 1


@pytest.mark.parametrize("flags", SCHEDULES)
@pytest.mark.parametrize("dtype,count,hi", [(np.complex128, 60, 1 << 17), (np.complex64, 80, 1 << 18)])
def test_batch_matches_single_plans(cb, dtype, count, hi, flags):
    import torch
    lengths = _lengths(cb, count, seed=count, hi=hi)
    b = cb.Batch(lengths, dtype, flags)
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(b.total) + 1j * rng.standard_normal(b.total)).astype(dtype)
    xd = torch.from_numpy(x).cuda()
    y = b.execute(xd).cpu().numpy()
    y2 = b.execute(xd).cpu().numpy()              # graph replay
    assert np.array_equal(y, y2)
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    for i, (o, n) in enumerate(zip(b.offsets, lengths)):
        seg = x[o:o + n]
        if dtype == np.complex128:
            ref = oracle.fft(seg)
            assert rel(y[o:o + n], ref) < bar64(ref, seg), (i, n)
        elif i % 4 == 0:                           # FP32 form vs the FP64 oracle
            ref = oracle.fft(seg.astype(np.complex128))
            assert rel(y[o:o + n], ref) < tol, (i, n)
    _check_launches(b, flags)
    b.close()


@pytest.mark.parametrize("flags", SCHEDULES)
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_batch_two_pass_members(cb, dtype, flags):
    """Lengths beyond one CTA run as column/row passes over a shared scratch
    (queue: tiles that wait for the previous stage of their transform);
    mixed with single-kernel lengths in the same batch."""
    import torch
    lengths = [16, 1 << 20, 531441, 4096, 999983, 30240, 65537, 300007, 1 << 19, 10007, 3]
    b = cb.Batch(lengths, dtype, flags)
    rng = np.random.default_rng(5)
    x = (rng.standard_normal(b.total) + 1j * rng.standard_normal(b.total)).astype(dtype)
    y = b.execute(torch.from_numpy(x).cuda()).cpu().numpy()
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    for o, n in zip(b.offsets, lengths):
        seg = x[o:o + n]
        ref = oracle.fft(seg.astype(np.complex128))
        if dtype == np.complex128:
            tol = bar64(ref, seg)
        assert rel(y[o:o + n], ref) < tol, n
    _check_launches(b, flags)
    b.close()


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_queue_scratch_ring_waits(cb, dtype, monkeypatch):
    """A 1 MB chunk budget puts nearly every two-pass transform in its own
    chunk, so chunks reuse the ring's slots and their first passes wait for
    earlier chunks; results must not change, nor the launch count."""
    import torch
    lengths = [1 << 17, 99991, 65536 * 3, 40000, 1 << 16, 77777, 250, 50000, 1 << 15, 33333] * 3
    rng = np.random.default_rng(9)
    monkeypatch.setenv("CFFT_SCRATCH_MB", "1")
    b = cb.Batch(lengths, dtype)
    monkeypatch.delenv("CFFT_SCRATCH_MB")
    x = (rng.standard_normal(b.total) + 1j * rng.standard_normal(b.total)).astype(dtype)
    xd = torch.from_numpy(x).cuda()
    y = b.execute(xd).cpu().numpy()
    ref_b = cb.Batch(lengths, dtype)               # default ring: few chunks
    y2 = ref_b.execute(xd).cpu().numpy()
    assert np.array_equal(y, y2)
    assert cb._lib.LIB.cfft_device_faults(1) == 0
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    for o, n in list(zip(b.offsets, lengths))[:10]:
        seg = x[o:o + n]
        ref = oracle.fft(seg.astype(np.complex128))
        if dtype == np.complex128:
            tol = bar64(ref, seg)
        assert rel(y[o:o + n], ref) < tol, n
    _check_launches(b, 0)
    b.close()
    ref_b.close()


@pytest.mark.parametrize("flags", SCHEDULES)
def test_batch_inverse_roundtrip_inplace(cb, flags):
    import torch
    lengths = _lengths(cb, 40, seed=7, hi=1 << 16)
    b = cb.Batch(lengths, np.complex128, flags)
    rng = np.random.default_rng(2)
    x = torch.from_numpy(rng.standard_normal(b.total) + 1j * rng.standard_normal(b.total)).cuda()
    y = b.execute(x)
    z = b.execute(y, cb.INVERSE, out=y)            # in place
    assert (torch.linalg.norm(z - x) / torch.linalg.norm(x)).item() < 1e-12
    b.close()


def test_batch_rejects_bad_lengths(cb):
    with pytest.raises(cb.CatabraError):
        cb.Batch([16, 0, 32], np.complex64)
