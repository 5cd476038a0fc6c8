"""Generate the committed golden fixtures for the 1D complex FFT.

Run from the repository root:  python tests/golden/make_golden.py

Inputs are seeded (numpy default_rng), outputs come from the CPU oracle
(oracle/catabra_oracle.c, a restatement of CatabraFFT.jl's algorithm).
Before writing, every output is cross-checked against numpy's pocketfft and,
for small n, against a direct DFT evaluated in extended precision; the
measured error against that exact reference is stored beside each case, so
the fixtures also record how far the reference algorithm itself sits from
the exact DFT (its Rader twiddles W = w^-k, prime.jl:36-37, and the mixed-
radix twiddle recurrence, mixed_radix.jl:30-41, accumulate rounding error).

Size classes follow the reference's test matrix (test/runtests.jl:9-33) and
the benchmark configurations (n = 4096, 30240, 10007, 2^16, 3^9).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

SEED = 20261203

# reference test matrix, sampled so the fixture file stays small
SIZES = (
    [10, 100, 1000, 10000]                      # mixed radix (runtests.jl:9-15)
    + [11, 13, 17, 19, 43, 89, 1721]            # Rader (runtests.jl:17-23)
    + [2 ** k for k in range(1, 13)]            # radix-2 family (runtests.jl:25-33)
    + [3 ** k for k in range(1, 8)]
    + [5 ** k for k in range(1, 6)]
    + [7 ** k for k in range(1, 5)]
    + [121, 257]                                # self-test size; Fermat prime
    + [30240, 10007]                            # plain mixed + Rader batch sizes
)


def exact_dft(x: np.ndarray, sign: int = -1) -> np.ndarray:
    """Direct DFT in numpy long double (80-bit on x86), row-blocked."""
    n = x.size
    xl = x.astype(np.clongdouble)
    k = np.arange(n, dtype=np.int64)
    out = np.empty(n, dtype=np.clongdouble)
    two_pi = np.longdouble(2) * np.arccos(np.longdouble(-1))
    blk = max(1, (1 << 22) // max(n, 1))
    for s in range(0, n, blk):
        rows = np.arange(s, min(n, s + blk), dtype=np.int64)
        idx = np.outer(rows, k) % n                      # exact integer phase
        ang = (sign * two_pi / n) * idx.astype(np.longdouble)
        out[s:s + rows.size] = (np.cos(ang) + 1j * np.sin(ang)) @ xl
    return out


def rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main() -> None:
    rng = np.random.default_rng(SEED)
    arrays = {}
    meta = []
    for n in SIZES:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = oracle.fft(x)
        yi = oracle.ifft(x)
        e_np = rel(y, np.fft.fft(x))
        e_ex = rel(y, exact_dft(x).astype(np.complex128)) if n <= 4096 else e_np
        assert e_np < 5e-12, (n, e_np)
        assert rel(yi, np.fft.ifft(x)) < 5e-12, n
        arrays[f"x_{n}"] = x
        arrays[f"fft_{n}"] = y
        if n <= 10000:
            arrays[f"ifft_{n}"] = yi
        meta.append((n, e_np, e_ex, oracle.describe(n)))
        print(f"n={n:6d} vs numpy {e_np:.2e}  vs exact {e_ex:.2e}  {oracle.describe(n)[:70]}")
    arrays["meta_n"] = np.array([m[0] for m in meta], dtype=np.int64)
    arrays["meta_err_numpy"] = np.array([m[1] for m in meta])
    arrays["meta_err_exact"] = np.array([m[2] for m in meta])
    arrays["meta_plan"] = np.array([m[3] for m in meta])
    np.savez_compressed(os.path.join(HERE, "c128_fixtures.npz"), **arrays)

    # ComplexF32 form: FP32 inputs; expected output is the FP64 oracle on the
    # same (FP32-representable) inputs, error bar 1e-5 relative L2.
    rng = np.random.default_rng(SEED + 1)
    arr32 = {}
    for n in [4096, 19683, 10007, 89, 1000]:
        x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
        arr32[f"x_{n}"] = x
        arr32[f"fft_{n}"] = oracle.fft(x.astype(np.complex128))
    np.savez_compressed(os.path.join(HERE, "c64_fixtures.npz"), **arr32)


if __name__ == "__main__":
    main()
