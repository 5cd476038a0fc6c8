"""Seeded synthetic workloads for the batched and served forms.

* batch_lengths: lengths log-uniform over [lo, hi]; half 7-smooth (the
  2^a 3^b 5^c 7^d number nearest the draw), half p * m with p a prime in
  (7, pmax] and m the 7-smooth cofactor nearest draw / p, kept in range.
* request_stream: Poisson arrivals at a given rate with lengths drawn the
  same way (share of prime-containing lengths configurable).
"""
from __future__ import annotations

import bisect
import math

import numpy as np


def _smooth_numbers(limit: int):
    out = []
    p2 = 1
    while p2 <= limit:
        p3 = p2
        while p3 <= limit:
            p5 = p3
            while p5 <= limit:
                p7 = p5
                while p7 <= limit:
                    out.append(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def _primes_upto(n: int):
    sieve = np.ones(n + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(n ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    return np.nonzero(sieve)[0]


_SMOOTH = _smooth_numbers(1 << 24)
_PRIMES = _primes_upto(65537)


def nearest_smooth(x: float, lo: int, hi: int) -> int:
    i = bisect.bisect_left(_SMOOTH, x)
    cands = [_SMOOTH[j] for j in (i - 1, i) if 0 <= j < len(_SMOOTH)]
    best = min(cands, key=lambda v: abs(math.log(v) - math.log(max(x, 1))))
    return int(min(max(best, lo), hi)) if lo <= best <= hi else int(
        min((v for v in _SMOOTH if lo <= v <= hi), key=lambda v: abs(v - x)))


def _draw(rng, lo, hi, prime_share, pmax):
    t = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    if rng.uniform() >= prime_share:
        return nearest_smooth(t, lo, hi)
    # prime factor p in (7, pmax], cofactor smooth
    top = min(pmax, max(11, int(t)))
    ps = _PRIMES[(_PRIMES > 7) & (_PRIMES <= top)]
    if len(ps) == 0:
        return nearest_smooth(t, lo, hi)
    p = int(ps[rng.integers(len(ps))])
    m = nearest_smooth(max(1.0, t / p), 1, max(1, hi // p))
    n = p * m
    while n < lo:
        n *= 2
    while n > hi and m > 1:
        m //= 2 if m % 2 == 0 else 1
        n = p * m
        if m == 1:
            break
    return int(min(max(n, lo), hi)) if n >= lo else int(p)


def batch_lengths(count: int, seed: int = 0, lo: int = 16, hi: int = 1 << 20,
                  prime_share: float = 0.5, pmax: int = 65537):
    rng = np.random.default_rng(seed)
    return [_draw(rng, lo, hi, prime_share, pmax) for _ in range(count)]


def request_stream(count: int, rate_hz: float, seed: int = 0, lo: int = 64, hi: int = 1 << 22,
                   prime_share: float = 0.2, pmax: int = 65537):
    """(arrival_time_s, n) pairs: Poisson arrivals at rate_hz."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=count)
    t = np.cumsum(gaps)
    return [(float(t[i]), _draw(rng, lo, hi, prime_share, pmax)) for i in range(count)]
