"""ctypes binding of libcatabra_b200.so (the C ABI in include/catabra_b200.h).

There is no CPU fallback: if the shared library is missing or does not load,
importing the package raises immediately.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcatabra_b200.so")

C128, C64, C32 = 0, 1, 2
FORWARD, INVERSE, BACKWARD = 0, 1, 2
NO_FLAG, MEASURE, ENCHANT, EXACT_TWIDDLES, BATCH_GROUPED = 0, 1, 2, 16, 32
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED = 0, 1, 2, 3, 4
SERVE_BATCHED, SERVE_DIRECT = 0, 1

# every symbol include/catabra_b200.h declares, with (restype, argtypes)
_i64, _vp, _ci, _cp = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p
SIGNATURES = {
    "cfft_plan_create": (_ci, [ctypes.POINTER(_vp), _i64, _i64, _ci, _ci]),
    "cfft_execute": (_ci, [_vp, _vp, _vp, _ci, _vp]),
    "cfft_execute_host": (_ci, [_vp, _vp, _vp, _ci]),
    "cfft_plan_destroy": (_ci, [_vp]),
    "cfft_fft": (_ci, [_i64, _i64, _ci, _ci, _vp, _vp, _ci, _vp]),
    "cfft_empty_cache": (_ci, []),
    "cfft_last_error": (_cp, []),
    "cfft_plan_describe": (_ci, [_vp, _cp, _ci]),
    "cfft_describe_strategy": (_ci, [_i64, _ci, _cp, _ci]),
    "cfft_plan_workspace_bytes": (_i64, [_vp]),
    "cfft_plan_launches": (_ci, [_vp]),
    "cfft_version": (_ci, []),
    "cfft_fft_twopass_noalloc": (_ci, [_i64, _i64, _ci, _vp, _vp, _ci, _vp]),
    "cfft_batch_create": (_ci, [ctypes.POINTER(_vp), _i64, ctypes.POINTER(_i64), _ci, _ci]),
    "cfft_batch_execute": (_ci, [_vp, _vp, _vp, _ci, _vp]),
    "cfft_batch_destroy": (_ci, [_vp]),
    "cfft_batch_elements": (_i64, [_vp]),
    "cfft_batch_launches": (_ci, [_vp]),
    "cfft_serve_create": (_ci, [ctypes.POINTER(_vp), _ci, _i64, _i64, _ci]),
    "cfft_serve_prepare": (_ci, [_vp, _i64, ctypes.POINTER(_i64)]),
    "cfft_serve_submit": (_ci, [_vp, _i64, _vp, _vp, _ci, ctypes.POINTER(_i64)]),
    "cfft_serve_query": (_ci, [_vp, _i64, ctypes.POINTER(_ci), ctypes.POINTER(ctypes.c_double)]),
    "cfft_serve_wait": (_ci, [_vp, _i64, ctypes.POINTER(ctypes.c_double)]),
    "cfft_serve_drain": (_ci, [_vp]),
    "cfft_serve_stats": (_ci, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "cfft_serve_destroy": (_ci, [_vp]),
    "cfft_plan_create_many": (_ci, [ctypes.POINTER(_vp), _i64, _i64, _ci, _ci, _i64, _i64, _i64, _i64]),
    "cfft_rfft_plan_create": (_ci, [ctypes.POINTER(_vp), _i64, _i64, _ci, _ci]),
    "cfft_rfft_execute": (_ci, [_vp, _vp, _vp, _vp]),
    "cfft_rfft_execute_inverse": (_ci, [_vp, _vp, _vp, _ci, _vp]),
    "cfft_rfft_execute_host": (_ci, [_vp, _vp, _vp, _ci]),
    "cfft_rfft_plan_destroy": (_ci, [_vp]),
    "cfft_wisdom_export": (_ci, [_cp]),
    "cfft_wisdom_import": (_ci, [_cp]),
    "cfft_wisdom_forget": (_ci, []),
    "cfft_wisdom_entries": (_i64, []),
    "cfft_debug_alloc_hook": (_i64, [_i64]),
    "cfft_device_faults": (_ci, [_ci]),
    "cfft_debug_wait_timeout": (_ci, [_ci]),
}


class CatabraError(RuntimeError):
    """A non-zero status from the C ABI, with cfft_last_error() text."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"catabra_b200 error {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python catabrafft.jl_b200/build.py` "
            "(this package has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = load()


def check(rc: int) -> None:
    if rc != OK:
        raise CatabraError(rc, LIB.cfft_last_error().decode(errors="replace"))
