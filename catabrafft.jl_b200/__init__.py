"""B200-native 1D complex FFT behind CatabraFFT.jl's public API.

Python mirror of the reference's API (src/CatabraFFT.jl), dispatching every
transform to libcatabra_b200.so (CUDA, sm_100a) through its C ABI:

    fft(x)            CatabraFFT.jl:65-72    forward, allocates the result
    ifft(x)           CatabraFFT.jl:88-101   inverse, scaled by 1/n
    bfft(x)           CatabraFFT.jl:103-115  inverse, unscaled
    fft_(x)           CatabraFFT.jl:46-49    in place (Julia's fft!)
    plan_fft(x, flag) CatabraFFT.jl:149-167  returns a Spell
    p * x, mul_(y,p,x) CatabraFFT.jl:186-196
    empty_cache()     CatabraFFT.jl:39-43
    NO_FLAG, MEASURE, ENCHANT                spells.jl:4-8

``x`` is a complex128 (ComplexF64) or complex64 (ComplexF32) array whose last
axis is transformed: 1-D of length n, or 2-D [batch, n] for a batch of
transforms.  numpy arrays (and CPU torch tensors) go through the host entry
point (copy in, transform, copy out); CUDA torch tensors stay on the device
and run on torch's current stream.  Inputs are never modified, except by
``fft_``.  Errors raise :class:`CatabraError` (a RuntimeError) or
ValueError/TypeError for arguments the reference would also reject.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from ._lib import (BACKWARD, BATCH_GROUPED, C32, C64, C128, ENCHANT, EXACT_TWIDDLES, FORWARD, INVERSE, MEASURE,
                   NO_FLAG, SERVE_BATCHED, SERVE_DIRECT, CatabraError, check)

FLAG = int
PLANNER_DEFAULT = NO_FLAG

__all__ = ["fft", "ifft", "bfft", "fft_", "plan_fft", "Spell", "mul_", "empty_cache", "Batch", "Server",
           "export_wisdom", "import_wisdom", "forget_wisdom", "wisdom_entries",
           "rfft", "irfft", "brfft", "plan_rfft", "plan_brfft", "RSpell", "plan_bfft", "plan_ifft",
           "plan_inv", "fftn", "ifftn", "fft2", "ifft2",
           "NO_FLAG", "MEASURE", "ENCHANT", "EXACT_TWIDDLES", "BATCH_GROUPED", "FLAG", "CatabraError",
           "describe_strategy", "version"]

_cache_lock = threading.Lock()
_plans: dict = {}


def version() -> int:
    return _lib.LIB.cfft_version()


def describe_strategy(n: int, dtype=np.complex128) -> str:
    """The planner's choice for length n (host logic only, no device work)."""
    buf = ctypes.create_string_buffer(512)
    check(_lib.LIB.cfft_describe_strategy(int(n), _dtype_code(dtype), buf, 512))
    return buf.value.decode()


def _dtype_code(dt) -> int:
    name = str(dt).replace("torch.", "")
    if name in ("complex128", "<class 'numpy.complex128'>"):
        return C128
    if name in ("complex64", "<class 'numpy.complex64'>"):
        return C64
    if name in ("complex32", "chalf"):        # torch.complex32: ComplexF16
        return C32
    raise TypeError(f"unsupported element type {dt}: expected complex128 or complex64")


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


class _Plan:
    """Owns one cfft_plan handle (device tables, scratch)."""

    def __init__(self, n, batch, dtype, flags, device):
        self.n, self.batch, self.dtype, self.flags, self.device = n, batch, dtype, flags, device
        h = ctypes.c_void_p()
        check(_lib.LIB.cfft_plan_create(ctypes.byref(h), n, batch, dtype, flags))
        self.handle = h

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        check(_lib.LIB.cfft_plan_describe(self.handle, buf, 512))
        return buf.value.decode()

    def launches(self) -> int:
        return _lib.LIB.cfft_plan_launches(self.handle)

    def workspace_bytes(self) -> int:
        return _lib.LIB.cfft_plan_workspace_bytes(self.handle)

    def destroy(self):
        if self.handle:
            _lib.LIB.cfft_plan_destroy(self.handle)
            self.handle = None


def _current_device(x=None) -> int:
    if x is not None and _is_torch(x) and x.is_cuda:
        return x.device.index
    return 0


def _get_plan(n, batch, dtype, flags, device) -> _Plan:
    key = (device, n, batch, dtype, flags)
    with _cache_lock:
        p = _plans.get(key)
        if p is None:
            p = _Plan(n, batch, dtype, flags, device)
            _plans[key] = p
        return p


def _shape(x):
    if x.ndim == 1:
        return x.shape[0], 1
    if x.ndim == 2:
        return x.shape[1], x.shape[0]
    raise ValueError("expected a vector of length n or a [batch, n] matrix")


def _run(x, direction: int, flags: int = NO_FLAG, out=None):
    if _is_torch(x):
        import torch
        if x.is_cuda:
            n, batch = _shape(x)
            if n < 1:
                raise ValueError("transform length must be >= 1")
            dt = _dtype_code(x.dtype)
            xc = x.contiguous()
            y = torch.empty_like(xc) if out is None else out
            if batch == 0:
                return y
            plan = _get_plan(n, batch, dt, flags, x.device.index)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            with torch.cuda.device(x.device):
                check(_lib.LIB.cfft_execute(plan.handle, ctypes.c_void_p(xc.data_ptr()),
                                            ctypes.c_void_p(y.data_ptr()), direction,
                                            ctypes.c_void_p(stream)))
            return y
        xn = x.detach().numpy()
        y = _run(xn, direction, flags)
        return torch.from_numpy(y)
    a = np.asarray(x)
    n, batch = _shape(a)
    if n < 1:
        raise ValueError("transform length must be >= 1")
    dt = _dtype_code(a.dtype)
    a = np.ascontiguousarray(a)
    y = np.empty_like(a) if out is None else out
    if batch == 0:
        return y
    plan = _get_plan(n, batch, dt, flags, 0)
    check(_lib.LIB.cfft_execute_host(plan.handle, a.ctypes.data_as(ctypes.c_void_p),
                                     y.ctypes.data_as(ctypes.c_void_p), direction))
    return y


def _run_axis(x, direction: int, axis: int):
    """Transform along one axis of an N-D array (the reference's `region`,
    ignored there at CatabraFFT.jl:169).  CUDA tensors use strided plans
    (cfft_plan_create_many): the axis has stride `inner`, the transforms of
    one outer index are `inner` apart by 1; host arrays are transposed on the
    host around the contiguous path."""
    nd = x.dim() if _is_torch(x) else np.ndim(x)
    if not -nd <= axis < nd:
        raise ValueError(f"axis {axis} out of range for a {nd}-D array")
    axis = axis % nd
    if axis == nd - 1:
        if nd <= 2:
            return _run(x, direction)
        if _is_torch(x):
            return _run(x.reshape(-1, x.shape[-1]), direction).reshape(x.shape)
        a = np.asarray(x)
        return _run(a.reshape(-1, a.shape[-1]), direction).reshape(a.shape)
    if _is_torch(x) and x.is_cuda:
        import torch
        xc = x.contiguous()
        shape = list(xc.shape)
        n = shape[axis]
        outer = int(np.prod(shape[:axis])) if axis else 1
        inner = int(np.prod(shape[axis + 1:]))
        y = torch.empty_like(xc)
        dt = _dtype_code(xc.dtype)
        e = 16 if dt == C128 else 8
        key = ("many", xc.device.index, n, inner, dt)
        with _cache_lock:
            h = _plans.get(key)
            if h is None:
                hp = ctypes.c_void_p()
                check(_lib.LIB.cfft_plan_create_many(ctypes.byref(hp), n, inner, dt, NO_FLAG, inner, 1, inner, 1))
                h = _ManyPlan(hp)
                _plans[key] = h
        stream = ctypes.c_void_p(torch.cuda.current_stream(xc.device).cuda_stream)
        with torch.cuda.device(xc.device):
            for o in range(outer):
                off = o * n * inner * e
                check(_lib.LIB.cfft_execute(h.handle, ctypes.c_void_p(xc.data_ptr() + off),
                                            ctypes.c_void_p(y.data_ptr() + off), direction, stream))
        return y
    if _is_torch(x):
        import torch
        return torch.from_numpy(_run_axis(x.detach().numpy(), direction, axis))
    a = np.moveaxis(np.asarray(x), axis, -1)
    return np.moveaxis(_run_axis(np.ascontiguousarray(a), direction, -1), -1, axis)


class _ManyPlan:
    def __init__(self, handle):
        self.handle = handle

    def destroy(self):
        if self.handle:
            _lib.LIB.cfft_plan_destroy(self.handle)
            self.handle = None


def fft(x, axis: int = -1):
    """Forward DFT along `axis` (default the last; CatabraFFT.fft)."""
    return _run(x, FORWARD) if axis == -1 and np.ndim(x) <= 2 and not (_is_torch(x) and x.dim() > 2) \
        else _run_axis(x, FORWARD, axis)


def ifft(x, axis: int = -1):
    """Inverse DFT scaled by 1/n (CatabraFFT.ifft: conj, fft, conj, /n)."""
    return _run(x, INVERSE) if axis == -1 and np.ndim(x) <= 2 and not (_is_torch(x) and x.dim() > 2) \
        else _run_axis(x, INVERSE, axis)


def bfft(x, axis: int = -1):
    """Unscaled inverse DFT (CatabraFFT.bfft)."""
    return _run(x, BACKWARD) if axis == -1 and np.ndim(x) <= 2 and not (_is_torch(x) and x.dim() > 2) \
        else _run_axis(x, BACKWARD, axis)


def fftn(x, axes=None):
    """Multi-dimensional DFT: one pass per axis (default all axes)."""
    nd = x.dim() if _is_torch(x) else np.ndim(x)
    for a in (range(nd) if axes is None else axes):
        x = _run_axis(x, FORWARD, a)
    return x


def ifftn(x, axes=None):
    nd = x.dim() if _is_torch(x) else np.ndim(x)
    for a in (range(nd) if axes is None else axes):
        x = _run_axis(x, INVERSE, a)
    return x


def fft2(x):
    return fftn(x, (-2, -1))


def ifft2(x):
    return ifftn(x, (-2, -1))


def fft_(x):
    """In-place forward DFT (Julia's fft!); returns x."""
    if _is_torch(x) and x.is_cuda:
        if not x.is_contiguous():
            raise ValueError("fft_ needs a contiguous tensor")
        _run(x, FORWARD, out=x)
        return x
    if not (isinstance(x, np.ndarray) and x.flags.c_contiguous and x.flags.writeable):
        raise ValueError("fft_ needs a writeable C-contiguous array")
    _run(x, FORWARD, out=x)
    return x


class Spell:
    """Plan object (the reference's Spell{T}, src/spells.jl:18-37).

    Holds n, datatype, flag and inverse like the reference; ``p * x`` and
    ``mul_(y, p, x)`` run the planned transform.  Unlike the reference, the
    flag is honoured at execution (spells.jl/kernel.jl:97 always ran the
    NO_FLAG function) and x is never overwritten.
    """

    def __init__(self, n: int, datatype, flag: int = NO_FLAG, batch: int = 1, device: int = 0,
                 direction: int = FORWARD):
        if n < 1:
            raise ValueError("transform length must be >= 1")
        self.n = int(n)
        self.datatype = datatype
        self.flag = int(flag)
        self.batch = int(batch)
        self.device = device
        self.direction = int(direction)
        self.inverse = None
        self._plan = _get_plan(self.n, self.batch, _dtype_code(datatype), self.flag, device)

    def describe(self) -> str:
        return self._plan.describe()

    def launches(self) -> int:
        return self._plan.launches()

    def _check(self, x):
        n, batch = _shape(x)
        if n != self.n or batch != self.batch:
            raise ValueError(f"plan is for n={self.n}, batch={self.batch}; got n={n}, batch={batch}")

    def __mul__(self, x):
        self._check(x)
        return _run(x, self.direction, self.flag)

    __matmul__ = __mul__

    def __call__(self, x):
        return self * x

    def adjoint(self) -> "Spell":
        """The adjoint (AbstractFFTs.adjoint_mul, CatabraFFT.jl:214-219): the
        DFT of the opposite sign with the same scaling -- bfft for a forward
        plan, fft for a bfft plan, fft / n for an ifft plan."""
        if self.direction == FORWARD:
            return Spell(self.n, self.datatype, self.flag, self.batch, self.device, BACKWARD)
        if self.direction == BACKWARD:
            return Spell(self.n, self.datatype, self.flag, self.batch, self.device, FORWARD)
        return _ScaledSpell(self, 1.0 / self.n)

    def __repr__(self):
        kind = {FORWARD: "fft", INVERSE: "ifft", BACKWARD: "bfft"}[self.direction]
        return f"Spell{{{self.datatype}}}({kind}, n={self.n}, flag={self.flag}, batch={self.batch})"


class _ScaledSpell:
    """c * fft: the adjoint of an ifft plan."""

    def __init__(self, p: Spell, c: float):
        self.p, self.c = p, c

    def __mul__(self, x):
        self.p._check(x)
        return _run(x, FORWARD, self.p.flag) * self.c


def plan_inv(p: Spell) -> Spell:
    """Inverse plan, cached on p (AbstractFFTs.plan_inv; the reference's
    CatabraFFT.jl:181-184): ifft for a forward plan, fft for an ifft plan,
    fft / n for a bfft plan."""
    if p.inverse is None:
        if p.direction == FORWARD:
            p.inverse = Spell(p.n, p.datatype, p.flag, p.batch, p.device, INVERSE)
        elif p.direction == INVERSE:
            p.inverse = Spell(p.n, p.datatype, p.flag, p.batch, p.device, FORWARD)
        else:
            p.inverse = _ScaledSpell(Spell(p.n, p.datatype, p.flag, p.batch, p.device, FORWARD), 1.0 / p.n)
    return p.inverse


def plan_bfft(x, flags: int = NO_FLAG) -> Spell:
    """Plan an unnormalised backward FFT (AbstractFFTs.plan_bfft; a stub in
    the reference, CatabraFFT.jl:173-177)."""
    n, batch = _shape(x)
    return Spell(n, x.dtype, flags, batch, _current_device(x), BACKWARD)


def plan_ifft(x, flags: int = NO_FLAG) -> Spell:
    """Plan an inverse FFT scaled by 1/n (AbstractFFTs.plan_ifft)."""
    n, batch = _shape(x)
    return Spell(n, x.dtype, flags, batch, _current_device(x), INVERSE)


def plan_fft(x, flags: int = NO_FLAG) -> Spell:
    """Plan a forward FFT for arrays shaped like x (CatabraFFT.plan_fft)."""
    if int(flags) & 3 not in (NO_FLAG, MEASURE, ENCHANT):
        raise ValueError("flags must be NO_FLAG, MEASURE or ENCHANT")
    n, batch = _shape(x)
    dev = _current_device(x)
    return Spell(n, x.dtype, flags, batch, dev)


def mul_(y, p: Spell, x):
    """y <- p * x (LinearAlgebra.mul! of the reference); returns y."""
    p._check(x)
    p._check(y)
    if _is_torch(x) and x.is_cuda:
        _run(x, FORWARD, p.flag, out=y)
        return y
    r = _run(x, FORWARD, p.flag)
    np.copyto(y, r)
    return y


class Batch:
    """Mixed-length batch (the batched form): transforms packed back to back.

    ``Batch(lengths, dtype)`` plans every distinct length once;
    ``b.execute(x)`` runs the whole batch on a CUDA torch tensor holding the
    packed transforms (1-D, ``sum(lengths)`` elements) as one graph launch on
    torch's current stream and returns the packed result.
    """

    def __init__(self, lengths, dtype=np.complex64, flags: int = 0):
        import ctypes as _ct
        self.lengths = [int(n) for n in lengths]
        self.dtype_code = _dtype_code(dtype)
        arr = (_ct.c_int64 * len(self.lengths))(*self.lengths)
        h = _ct.c_void_p()
        check(_lib.LIB.cfft_batch_create(_ct.byref(h), len(self.lengths), arr, self.dtype_code, int(flags)))
        self.handle = h
        self.total = int(_lib.LIB.cfft_batch_elements(h))
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths)[:-1]]).astype(np.int64)

    def launches(self) -> int:
        return int(_lib.LIB.cfft_batch_launches(self.handle))

    def execute(self, x, direction: int = FORWARD, out=None):
        import torch
        if not (_is_torch(x) and x.is_cuda and x.dim() == 1 and x.numel() == self.total):
            raise ValueError(f"expected a 1-D CUDA tensor of {self.total} elements")
        if _dtype_code(x.dtype) != self.dtype_code:
            raise TypeError("element type does not match the batch")
        xc = x.contiguous()
        y = torch.empty_like(xc) if out is None else out
        stream = torch.cuda.current_stream(x.device).cuda_stream
        check(_lib.LIB.cfft_batch_execute(self.handle, ctypes.c_void_p(xc.data_ptr()),
                                          ctypes.c_void_p(y.data_ptr()), int(direction),
                                          ctypes.c_void_p(stream)))
        return y

    def close(self):
        if getattr(self, "handle", None):
            _lib.LIB.cfft_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving form: requests submitted one at a time, batched on the device.

    ``Server(dtype, mode=SERVE_BATCHED, max_inflight_bytes=0)``;
    ``t = s.submit(x, y, direction)`` queues the transform of the 1-D CUDA
    tensor ``x`` into ``y`` (same length and type) and returns a ticket;
    ``s.wait(t)`` blocks until it is done and returns its latency in
    microseconds.  The tensors must stay alive until the request is done.
    ``mode=SERVE_DIRECT`` launches each request on arrival instead (the
    per-request path).
    """

    def __init__(self, dtype=np.complex64, mode: int = SERVE_BATCHED, max_inflight_bytes: int = 0,
                 max_requests: int = 0):
        h = ctypes.c_void_p()
        self.dtype_code = _dtype_code(dtype)
        check(_lib.LIB.cfft_serve_create(ctypes.byref(h), self.dtype_code, int(max_inflight_bytes),
                                         int(max_requests), int(mode)))
        self.handle = h

    def prepare(self, lengths) -> None:
        arr = (ctypes.c_int64 * len(lengths))(*[int(n) for n in lengths])
        check(_lib.LIB.cfft_serve_prepare(self.handle, len(lengths), arr))

    def submit(self, x, y, direction: int = FORWARD) -> int:
        if not (_is_torch(x) and x.is_cuda and x.is_contiguous() and y.is_contiguous()
                and x.numel() == y.numel()):
            raise ValueError("expected contiguous CUDA tensors of equal length")
        if _dtype_code(x.dtype) != self.dtype_code or _dtype_code(y.dtype) != self.dtype_code:
            raise TypeError("element type does not match the server")
        return self.submit_ptr(x.numel(), x.data_ptr(), y.data_ptr(), direction)

    def submit_ptr(self, n: int, d_in: int, d_out: int, direction: int = FORWARD) -> int:
        t = ctypes.c_int64()
        check(_lib.LIB.cfft_serve_submit(self.handle, int(n), ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                         int(direction), ctypes.byref(t)))
        return t.value

    def query(self, ticket: int):
        """Latency in microseconds once done, else None."""
        done, lat = ctypes.c_int(), ctypes.c_double()
        check(_lib.LIB.cfft_serve_query(self.handle, int(ticket), ctypes.byref(done), ctypes.byref(lat)))
        return lat.value if done.value else None

    def wait(self, ticket: int) -> float:
        lat = ctypes.c_double()
        check(_lib.LIB.cfft_serve_wait(self.handle, int(ticket), ctypes.byref(lat)))
        return lat.value

    def drain(self) -> None:
        check(_lib.LIB.cfft_serve_drain(self.handle))

    def stats(self):
        r, b, l = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(_lib.LIB.cfft_serve_stats(self.handle, ctypes.byref(r), ctypes.byref(b), ctypes.byref(l)))
        return {"requests": r.value, "batches": b.value, "launches": l.value}

    def close(self):
        if getattr(self, "handle", None):
            check(_lib.LIB.cfft_serve_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ real input
def _real_code(dt) -> int:
    name = str(dt).replace("torch.", "")
    if name in ("float64", "<class 'numpy.float64'>"):
        return C128
    if name in ("float32", "<class 'numpy.float32'>"):
        return C64
    raise TypeError(f"unsupported real element type {dt}: expected float64 or float32")


_rplans = {}


class _RPlan:
    """Owns one cfft_rplan (n reals <-> n/2 + 1 complex, batch transforms)."""

    def __init__(self, n, batch, dtype, flags):
        h = ctypes.c_void_p()
        check(_lib.LIB.cfft_rfft_plan_create(ctypes.byref(h), n, batch, dtype, flags))
        self.handle, self.n, self.batch, self.dtype = h, n, batch, dtype

    def destroy(self):
        if self.handle:
            _lib.LIB.cfft_rfft_plan_destroy(self.handle)
            self.handle = None


def _get_rplan(n, batch, dtype, flags, device):
    key = (device, n, batch, dtype, flags)
    with _cache_lock:
        p = _rplans.get(key)
        if p is None:
            p = _RPlan(n, batch, dtype, flags)
            _rplans[key] = p
        return p


def _rrun(x, n, direction, flags=NO_FLAG):
    """direction FORWARD: reals [.., n] -> complex [.., n//2+1]; else the reverse."""
    fwd = direction == FORWARD
    if _is_torch(x) and x.is_cuda:
        import torch
        xc = x.contiguous()
        rows = 1 if xc.dim() == 1 else xc.shape[0]
        dt = _real_code(xc.dtype) if fwd else _dtype_code(xc.dtype)
        rdt = torch.float64 if dt == C128 else torch.float32
        cdt = torch.complex128 if dt == C128 else torch.complex64
        shp = (n // 2 + 1,) if fwd else (n,)
        if xc.dim() == 2:
            shp = (rows,) + shp
        y = torch.empty(shp, dtype=cdt if fwd else rdt, device=xc.device)
        plan = _get_rplan(n, rows, dt, flags, xc.device.index)
        stream = ctypes.c_void_p(torch.cuda.current_stream(xc.device).cuda_stream)
        with torch.cuda.device(xc.device):
            if fwd:
                check(_lib.LIB.cfft_rfft_execute(plan.handle, ctypes.c_void_p(xc.data_ptr()),
                                                 ctypes.c_void_p(y.data_ptr()), stream))
            else:
                check(_lib.LIB.cfft_rfft_execute_inverse(plan.handle, ctypes.c_void_p(xc.data_ptr()),
                                                         ctypes.c_void_p(y.data_ptr()), direction, stream))
        return y
    if _is_torch(x):
        import torch
        return torch.from_numpy(_rrun(x.detach().numpy(), n, direction, flags))
    a = np.ascontiguousarray(np.asarray(x))
    if a.ndim not in (1, 2):
        raise ValueError("expected a vector or a [batch, n] matrix")
    rows = 1 if a.ndim == 1 else a.shape[0]
    dt = _real_code(a.dtype) if fwd else _dtype_code(a.dtype)
    if fwd and a.shape[-1] != n:
        raise ValueError("length mismatch")
    if not fwd and a.shape[-1] != n // 2 + 1:
        raise ValueError(f"expected {n // 2 + 1} spectrum values for n = {n}")
    shp = (n // 2 + 1,) if fwd else (n,)
    if a.ndim == 2:
        shp = (rows,) + shp
    y = np.empty(shp, dtype=(np.complex128 if dt == C128 else np.complex64) if fwd
                 else (np.float64 if dt == C128 else np.float32))
    plan = _get_rplan(n, rows, dt, flags, 0)
    check(_lib.LIB.cfft_rfft_execute_host(plan.handle, a.ctypes.data_as(ctypes.c_void_p),
                                          y.ctypes.data_as(ctypes.c_void_p), direction))
    return y


def rfft(x):
    """Real-input forward DFT: n reals -> n//2 + 1 complex (AbstractFFTs.rfft)."""
    n = x.shape[-1]
    if n < 1:
        raise ValueError("transform length must be >= 1")
    return _rrun(x, n, FORWARD)


def irfft(X, n: int):
    """Inverse of rfft for a Hermitian spectrum of n//2 + 1 values, scaled 1/n."""
    return _rrun(X, int(n), INVERSE)


def brfft(X, n: int):
    """Unscaled irfft (AbstractFFTs.brfft)."""
    return _rrun(X, int(n), BACKWARD)


class RSpell:
    """Real-input plan (the reference's plan_rfft / plan_brfft stubs,
    src/CatabraFFT.jl:199-209): ``p * x`` runs rfft (or, for a plan made by
    plan_brfft, brfft) with the plan's flag."""

    def __init__(self, n: int, flag: int = NO_FLAG, backward: bool = False):
        self.n, self.flag, self.backward = int(n), int(flag), backward

    def __mul__(self, x):
        return _rrun(x, self.n, BACKWARD if self.backward else FORWARD, self.flag)


def plan_rfft(x, flag: int = NO_FLAG) -> RSpell:
    return RSpell(np.asarray(x).shape[-1] if not _is_torch(x) else x.shape[-1], flag)


def plan_brfft(X, d: int, flag: int = NO_FLAG) -> RSpell:
    return RSpell(d, flag, backward=True)


def export_wisdom(path) -> None:
    """Save the shapes MEASURE/ENCHANT chose in this process (spells.jl's
    serialisable-Spell intent)."""
    check(_lib.LIB.cfft_wisdom_export(str(path).encode()))


def import_wisdom(path) -> None:
    """Merge a wisdom file: later MEASURE/ENCHANT plans of those keys skip timing."""
    check(_lib.LIB.cfft_wisdom_import(str(path).encode()))


def forget_wisdom() -> None:
    check(_lib.LIB.cfft_wisdom_forget())


def wisdom_entries() -> int:
    return int(_lib.LIB.cfft_wisdom_entries())


def empty_cache() -> None:
    """Free every cached plan and its device memory (CatabraFFT.empty_cache)."""
    with _cache_lock:
        for p in _plans.values():
            p.destroy()
        _plans.clear()
        for p in _rplans.values():
            p.destroy()
        _rplans.clear()
    check(_lib.LIB.cfft_empty_cache())
