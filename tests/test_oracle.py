"""CPU oracle checks: the restatement against the reference's test contract.

The reference (test/runtests.jl) checks CatabraFFT against FFTW at
rtol = sqrt(eps).  Julia is absent here, so the oracle is pinned against
numpy's pocketfft (the FFTW stand-in), an extended-precision direct DFT and
the committed golden fixtures.
"""
import numpy as np
import pytest

import oracle


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_golden_fixtures_reproduce(golden128):
    for n in golden128["meta_n"]:
        n = int(n)
        x = golden128[f"x_{n}"]
        assert rel(oracle.fft(x), golden128[f"fft_{n}"]) < 1e-15, n
        if f"ifft_{n}" in golden128:
            assert rel(oracle.ifft(x), golden128[f"ifft_{n}"]) < 1e-15, n


def test_golden_vs_exact_recorded(golden128):
    # the reference algorithm sits within 1e-12 of the exact DFT on every
    # fixture size (largest: Rader 10007 at ~7e-13)
    assert np.all(golden128["meta_err_exact"] < 1e-12)
    assert np.all(golden128["meta_err_numpy"] < 1e-12)


@pytest.mark.parametrize("n", [10, 100, 1000, 10 ** 4, 10 ** 5])
def test_mixed_radix_vs_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert rel(oracle.fft(x), np.fft.fft(x)) < 1.5e-8      # runtests.jl rtol
    assert rel(oracle.ifft(x), np.fft.ifft(x)) < 1.5e-8


@pytest.mark.parametrize("n", [11, 13, 17, 19, 43, 89, 1721, 257, 65537])
def test_rader_vs_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert rel(oracle.fft(x), np.fft.fft(x)) < 1.5e-8
    assert rel(oracle.fft(x, precision="f32"), np.fft.fft(x)) < 3.5e-4


@pytest.mark.parametrize("b,maxexp", [(2, 20), (3, 13), (5, 10), (7, 8)])
def test_pure_radix_families(b, maxexp):
    rng = np.random.default_rng(b)
    for e in range(1, maxexp + 1):
        n = b ** e
        if n > 2 ** 20:
            continue
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert rel(oracle.fft(x), np.fft.fft(x)) < 1e-13, n


def test_self_roundtrip_f64_f32():
    rng = np.random.default_rng(7)
    for n in [89, 121, 2 ** 10, 2 ** 11, 3 ** 7, 5 ** 6, 10 ** 4]:   # runtests.jl:39-46
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert rel(oracle.ifft(oracle.fft(x)), x) < 1e-13
        x32 = x.astype(np.complex64)
        back = oracle.ifft(oracle.fft(x32, precision="f32"), precision="f32")
        assert rel(back, x32) < 3.5e-4


def test_bfft_is_unnormalised_inverse():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(360) + 1j * rng.standard_normal(360)
    assert rel(oracle.bfft(x), np.fft.ifft(x) * 360) < 1e-13


def test_plan_choices_match_reference_heuristics():
    # kernel.jl:72-92 strategy, radix_plan.jl greedy, kernel.jl:169-191 factors
    assert oracle.describe(4096) == "radix(8,8,8,8)"
    assert oracle.describe(65536) == "radix(8,8,8,8,8,2)"
    assert oracle.describe(19683) == "radix(9,9,9,9,3)"
    assert oracle.describe(30240).startswith("mixed(32,945)[mixed(27,35)")
    assert oracle.describe(10007).startswith("rader(10007,g=5)[mixed(2,5003)")
    assert oracle.find_closest_factors(30240) == (32, 945)
    assert oracle.find_closest_factors(945) == (27, 35)
    assert oracle.find_closest_factors(35) == (7, 5)
    assert oracle.find_closest_factors(10006) == (2, 5003)
    assert oracle.find_closest_factors(2501) == (41, 61)        # sqrt fallback
    assert oracle.find_closest_factors(10007) == (1, 10007)
    assert oracle.rader_generator(10007) == 5
    assert oracle.rader_generator(65537) == 3


def test_codelets_in_explicit_plans():
    # every codelet, layered and last, through explicit Stockham plans
    rng = np.random.default_rng(11)
    for radices in [[16, 16], [16, 8, 2], [8, 4, 2], [9, 3], [3, 9], [5, 5, 5], [7, 7],
                    [4, 4, 4], [2, 2, 2, 2], [3, 3, 3]]:
        n = int(np.prod(radices))
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert rel(oracle.radix_plan_exec(x, radices), np.fft.fft(x)) < 1e-14, radices


def test_rader_clobber_mode_differs_only_after_first_call():
    # prime.jl:61 hands the captured W to a pure-radix F with >= 3 passes
    rng = np.random.default_rng(5)
    x = rng.standard_normal(257) + 1j * rng.standard_normal(257)
    good = np.fft.fft(x)
    try:
        oracle.set_rader_mode(True)
        first = oracle.fft(x)
        second = oracle.fft(x)
    finally:
        oracle.set_rader_mode(False)
    assert rel(first, good) < 1e-13
    assert rel(second, good) > 1e-3            # W destroyed by the first call
    assert rel(oracle.fft(x), good) < 1e-13     # fixed mode


def test_batch_threads_identical():
    rng = np.random.default_rng(9)
    x = rng.standard_normal((16, 1000)) + 1j * rng.standard_normal((16, 1000))
    a = oracle.fft(x, threads=1)
    b = oracle.fft(x, threads=4)
    assert np.array_equal(a, b)
