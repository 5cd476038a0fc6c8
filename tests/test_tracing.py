"""NVTX ranges around the C-ABI entry points.

The library wraps plan creation, execution, the host pipeline, the batched
and serving forms and the wisdom files in NVTX ranges of the domain
"catabra_b200" (the reference only prints: src/radix_exec.jl:91,179-183,
src/kernel.jl:115).  A tiny NVTX injection library (tests/nvtx_probe.c,
built here with gcc) records what a profiler would see; a child process
loads the product with NVTX_INJECTION64_PATH pointing at it, makes calls
and returns the record.  The CPU test uses calls that need no device (a
wisdom export, and a plan creation that fails without a GPU); the GPU test
checks that an execution's range carries the plan's description.
"""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "catabrafft.jl_b200", "libcatabra_b200.so")

CHILD = r"""
import ctypes, json, sys
probe = ctypes.CDLL(sys.argv[1])
lib = ctypes.CDLL(sys.argv[2])
lib.cfft_plan_describe.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
lib.cfft_plan_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
lib.cfft_execute.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p]
lib.cfft_wisdom_export.argtypes = [ctypes.c_char_p]
out = {"export": lib.cfft_wisdom_export(sys.argv[3].encode())}
h = ctypes.c_void_p()
out["create"] = lib.cfft_plan_create(ctypes.byref(h), 4096, 2, 0, 0)
if sys.argv[4] == "gpu":
    import torch
    x = torch.zeros(2, 4096, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    out["exec"] = lib.cfft_execute(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), 0, None)
    torch.cuda.synchronize()
    buf = ctypes.create_string_buffer(256)
    lib.cfft_plan_describe(h, buf, 256)
    out["desc"] = buf.value.decode()
buf = ctypes.create_string_buffer(1 << 16)
probe.nvtx_probe_dump(buf, 1 << 16)
out["log"] = buf.value.decode()
print(json.dumps(out))
"""


def _trace(tmp_path, mode):
    probe = tmp_path / "nvtx_probe.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-I/usr/local/cuda/include",
                    os.path.join(HERE, "nvtx_probe.c"), "-o", str(probe)], check=True)
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(probe))
    r = subprocess.run([sys.executable, "-c", CHILD, str(probe), LIB, str(tmp_path / "w.txt"), mode],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    lines = out["log"].splitlines()
    depth = 0
    for ln in lines:                       # every push has its pop, in order
        depth += ln.startswith("push ") - (ln == "pop")
        assert depth >= 0, lines
    assert depth == 0, lines
    return out, lines


def test_ranges_on_host_entry_points(tmp_path):
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    out, lines = _trace(tmp_path, "cpu")
    assert out["export"] == 0
    assert lines[0] == "domain catabra_b200"
    assert "push wisdom_export" in lines
    assert "push plan_create n=4096 batch=2 dtype=0 flags=0" in lines


@pytest.mark.gpu
def test_execute_range_names_the_plan(tmp_path):
    out, lines = _trace(tmp_path, "gpu")
    assert out["create"] == 0 and out["exec"] == 0
    assert "push " + out["desc"] in lines
