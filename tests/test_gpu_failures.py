"""Failure paths: allocations that fail as out of memory, and a device-side
wait that runs out.

The reference has no failure handling beyond Julia exceptions
(src/kernel.jl:113,187; src/prime.jl:6,27,43).  Here every create entry
point must return CFFT_ERR_NOMEM with a message when an allocation fails,
and release whatever it had already allocated.  The failure is injected on
the host (cfft_debug_alloc_hook makes the library's own allocations report
out-of-memory from the nth on); nothing faults the device.  A leak shows as
a live-allocation count (the library counts its own device and pinned host
allocations) or free device memory that does not return to its baseline.
The kernels' bounded waits are exercised on an mbarrier that nothing
completes (cfft_debug_wait_timeout): the wait gives up, the device fault
word reports it, and the context stays usable.
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
    m = load()
    yield m
    m._lib.LIB.cfft_debug_alloc_hook(0)


def _baseline(cb):
    """Live allocations and free device memory with every cache dropped."""
    import torch
    torch.cuda.synchronize()
    cb.empty_cache()
    torch.cuda.synchronize()
    return cb._lib.LIB.cfft_debug_alloc_hook(0), torch.cuda.mem_get_info()[0]


def _assert_released(cb, base, what):
    live, free = _baseline(cb)
    assert live == base[0], (what, live, base[0])
    assert abs(free - base[1]) <= (4 << 20), (what, free, base[1])


def _sweep(cb, create, destroy, what, limit=200):
    """Fail the kth allocation for k = 1, 2, ... until a create succeeds;
    every failing create must report CFFT_ERR_NOMEM and leak nothing."""
    lib = cb._lib.LIB
    base = _baseline(cb)
    failures = 0
    for k in range(1, limit):
        lib.cfft_debug_alloc_hook(k)
        rc, handle = create()
        lib.cfft_debug_alloc_hook(0)
        if rc == cb._lib.OK:
            destroy(handle)
            _assert_released(cb, base, (what, "success"))
            return failures
        assert rc == cb._lib.ERR_NOMEM, (what, k, rc, lib.cfft_last_error())
        assert lib.cfft_last_error(), (what, k)
        _assert_released(cb, base, (what, k))
        failures += 1
    raise AssertionError(f"{what}: still failing after {limit} injected allocations")


@pytest.mark.parametrize("n,batch,dtype", [(1 << 20, 6, 0), (10007, 8, 0), (30240, 3, 1), (4096, 5, 0),
                                           (999983, 2, 0), (3 ** 9, 4, 2)])
def test_plan_create_out_of_memory_releases_everything(cb, n, batch, dtype):
    lib = cb._lib.LIB

    def create():
        h = ctypes.c_void_p()
        rc = lib.cfft_plan_create(ctypes.byref(h), n, batch, dtype, cb.NO_FLAG)
        return rc, h

    failures = _sweep(cb, create, lambda h: lib.cfft_plan_destroy(h), ("plan", n))
    assert failures >= 1                      # at least one allocation was exercised


def test_measure_plan_out_of_memory(cb):
    # MEASURE allocates a timing buffer and builds several candidates
    lib = cb._lib.LIB

    def create():
        h = ctypes.c_void_p()
        return lib.cfft_plan_create(ctypes.byref(h), 30240, 2, cb.C128, cb.MEASURE), h

    assert _sweep(cb, create, lambda h: lib.cfft_plan_destroy(h), "measure") >= 1
    cb.forget_wisdom()


def test_batch_create_out_of_memory(cb):
    lib = cb._lib.LIB
    lengths = (ctypes.c_int64 * 6)(4096, 30240, 10007, 1 << 20, 65537, 17)

    def create():
        h = ctypes.c_void_p()
        return lib.cfft_batch_create(ctypes.byref(h), 6, lengths, cb.C64, 0), h

    assert _sweep(cb, create, lambda h: lib.cfft_batch_destroy(h), "batch", limit=400) >= 1


def test_host_entry_out_of_memory(cb):
    """The host entry allocates its staging pipeline on first use; a failure
    there is reported and the plan stays usable once memory is back."""
    lib = cb._lib.LIB
    base = _baseline(cb)
    n, batch = 4096, 4
    h = ctypes.c_void_p()
    cb.check(lib.cfft_plan_create(ctypes.byref(h), n, batch, cb.C128, cb.NO_FLAG))
    rng = np.random.default_rng(3)
    x = rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))
    y = np.empty_like(x)
    vp = ctypes.c_void_p
    lib.cfft_debug_alloc_hook(1)
    rc = lib.cfft_execute_host(h, vp(x.ctypes.data), vp(y.ctypes.data), cb.FORWARD)
    lib.cfft_debug_alloc_hook(0)
    assert rc == cb._lib.ERR_NOMEM, (rc, lib.cfft_last_error())
    cb.check(lib.cfft_execute_host(h, vp(x.ctypes.data), vp(y.ctypes.data), cb.FORWARD))
    errs = [np.linalg.norm(y[b] - oracle.fft(x[b])) / np.linalg.norm(y[b]) for b in range(batch)]
    assert max(errs) < 1e-12
    lib.cfft_plan_destroy(h)
    _assert_released(cb, base, "host entry")


def test_serve_admission_out_of_memory(cb):
    """A request whose launch slot must grow its scratch fails with
    CFFT_ERR_NOMEM when that allocation fails; the server keeps serving, and
    the same request succeeds once allocations succeed again."""
    import torch
    lib = cb._lib.LIB
    n = 1 << 21                                    # a two-pass length: needs slot scratch
    srv = cb.Server(np.complex64)
    srv.prepare([n, 4096])
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.complex(torch.randn(n, device="cuda", generator=g), torch.randn(n, device="cuda", generator=g))
    y = torch.empty_like(x)
    lib.cfft_debug_alloc_hook(1)
    t = srv.submit(x, y)
    with pytest.raises(cb.CatabraError):
        srv.wait(t)
    lib.cfft_debug_alloc_hook(0)
    small = x[:4096].clone()
    ys = torch.empty_like(small)
    srv.wait(srv.submit(small, ys))                # a request that needs no new memory
    srv.wait(srv.submit(x, y))                     # the failed one, now admitted
    srv.close()
    xh = x.cpu().numpy().astype(np.complex128)
    ref = oracle.fft(xh)
    assert np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-5
    ref_s = oracle.fft(xh[:4096])
    assert np.linalg.norm(ys.cpu().numpy() - ref_s) / np.linalg.norm(ref_s) < 1e-5


def test_empty_cache_while_server_is_live(cb):
    """Dropping the plan and table caches while a server holds plans (and has
    requests in flight) must not free anything the server still uses."""
    import torch
    lengths = [4096, 30240, 10007, 1 << 18, 65537]
    srv = cb.Server(np.complex128)
    srv.prepare(lengths)
    rng = np.random.default_rng(12)
    xs = [rng.standard_normal(n) + 1j * rng.standard_normal(n) for n in lengths]
    xd = [torch.from_numpy(v).cuda() for v in xs]
    ys = [torch.empty_like(v) for v in xd]
    first = [srv.submit(a, b) for a, b in zip(xd, ys)]
    cb.empty_cache()                               # while those requests may still run
    for t in first:
        srv.wait(t)
    ys2 = [torch.empty_like(v) for v in xd]
    for t in [srv.submit(a, b) for a, b in zip(xd, ys2)]:
        srv.wait(t)
    srv.close()
    for v, a, b in zip(xs, ys, ys2):
        ref = oracle.fft(v)
        bar = max(1e-12, np.linalg.norm(ref - np.fft.fft(v)) / np.linalg.norm(ref) + 1e-12)
        assert np.linalg.norm(a.cpu().numpy() - ref) / np.linalg.norm(ref) < bar
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_bounded_wait_times_out_without_a_fault(cb):
    """A kernel's bounded wait on an mbarrier that nothing completes gives up
    after its poll limit, records the device fault bit and returns: the host
    reads the bit, clears it, and the context keeps working."""
    lib = cb._lib.LIB
    assert lib.cfft_device_faults(1) >= 0
    assert lib.cfft_device_faults(0) == 0
    cb.check(lib.cfft_debug_wait_timeout(1000))
    assert lib.cfft_device_faults(1) & 1
    assert lib.cfft_device_faults(0) == 0
    x = np.ones(4096, dtype=np.complex128)
    assert abs(cb.fft(x)[0] - 4096) < 1e-9                # the context is still usable
    with pytest.raises(cb.CatabraError):
        cb.check(lib.cfft_debug_wait_timeout(0))
