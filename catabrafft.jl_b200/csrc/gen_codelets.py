"""Symbolic codelet generator: emits straight-line CUDA C DFT butterflies.

This re-targets the idea of CatabraFFT.jl's offline generators
(src/symbfftkernel.jl:17-60 ``recfft`` and src/radix_factory.jl:129-283
``recfft2``): a radix-r DFT is unrolled symbolically into straight-line code
and the twiddle constants are recognised and folded.  Differences from the
reference generators:

* it emits CUDA C device functions (``codelets.cuh``) operating in place on a
  register array ``V a[R]`` (V = double2 or float2) instead of Julia source;
* composite radices recurse by decimation in time over their smallest prime
  factor (radix_factory.jl only handles powers of two); odd prime radices use
  the symmetric-pair formulation the reference's radix-3/5/7 codelets use
  (radix_5_codelets.jl:14-23, radix_7_codelets.jl:15-25);
* constants are evaluated with exact rational angles in 50-digit decimal
  arithmetic and rounded once to binary64, then converted to the codelet's
  real type; +-1, +-i and (+-1 +- i)/sqrt(2) are folded into adds/swaps as in
  radix_factory.jl:56-65.

Run:  python gen_codelets.py  (rewrites codelets.cuh next to this file).
The generated file is committed; the build does not need Python.
"""
from __future__ import annotations

import os
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 60
RADICES = [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 15, 16, 18]


def _pi() -> Decimal:
    # Chudnovsky would be overkill; Machin's formula at 60 digits
    getcontext().prec = 70

    def arctan_inv(x):
        x = Decimal(x)
        total, term, n, sign = Decimal(0), 1 / x, 1, 1
        x2 = x * x
        while True:
            t = term / n
            if t < Decimal(10) ** -68:
                break
            total += sign * t
            term /= x2
            n += 2
            sign = -sign
        return total

    pi = 16 * arctan_inv(5) - 4 * arctan_inv(239)
    getcontext().prec = 60
    return +pi


PI = _pi()


def _cos_sin(frac: Fraction):
    """cos/sin of 2*pi*frac with Taylor series in Decimal (|angle| reduced)."""
    f = frac - (frac.numerator // frac.denominator)        # [0, 1)
    ang = 2 * PI * Decimal(f.numerator) / Decimal(f.denominator)
    if ang > PI:
        ang -= 2 * PI
    getcontext().prec = 70
    x2 = ang * ang
    c, s = Decimal(0), Decimal(0)
    term_c, term_s = Decimal(1), ang
    k = 0
    while True:
        c += term_c
        s += term_s
        term_c *= -x2 / ((2 * k + 1) * (2 * k + 2))
        term_s *= -x2 / ((2 * k + 2) * (2 * k + 3))
        k += 1
        if abs(term_c) < Decimal(10) ** -66 and abs(term_s) < Decimal(10) ** -66:
            break
    getcontext().prec = 60
    return +c, +s


def lit(d: Decimal) -> str:
    """Decimal -> correctly rounded binary64 literal."""
    return repr(float(d))


class Emitter:
    def __init__(self):
        self.lines = []
        self.k = 0

    def tmp(self):
        self.k += 1
        return f"t{self.k}"

    def assign(self, re: str, im: str) -> str:
        t = self.tmp()
        self.lines.append(f"    const V {t} = mk<V>({re}, {im});")
        return t

    def add(self, a, b):
        return self.assign(f"{a}.x + {b}.x", f"{a}.y + {b}.y")

    def sub(self, a, b):
        return self.assign(f"{a}.x - {b}.x", f"{a}.y - {b}.y")

    def twiddle(self, a: str, frac: Fraction) -> str:
        """a * exp(-2*pi*i*frac) with constant folding."""
        f = frac - (frac.numerator // frac.denominator)
        if f == 0:
            return a
        if f == Fraction(1, 2):
            return self.assign(f"-{a}.x", f"-{a}.y")
        if f == Fraction(1, 4):                 # -i
            return self.assign(f"{a}.y", f"-{a}.x")
        if f == Fraction(3, 4):                 # +i
            return self.assign(f"-{a}.y", f"{a}.x")
        h = "R(0.7071067811865476)"
        if f == Fraction(1, 8):                 # (1 - i)/sqrt2
            return self.assign(f"{h} * ({a}.x + {a}.y)", f"{h} * ({a}.y - {a}.x)")
        if f == Fraction(3, 8):                 # (-1 - i)/sqrt2
            return self.assign(f"{h} * ({a}.y - {a}.x)", f"-{h} * ({a}.x + {a}.y)")
        if f == Fraction(5, 8):                 # (-1 + i)/sqrt2
            return self.assign(f"-{h} * ({a}.x + {a}.y)", f"{h} * ({a}.x - {a}.y)")
        if f == Fraction(7, 8):                 # (1 + i)/sqrt2
            return self.assign(f"{h} * ({a}.x - {a}.y)", f"{h} * ({a}.x + {a}.y)")
        c, s = _cos_sin(f)
        # (a.x + i a.y)(c - i s) = (a.x c + a.y s) + i(a.y c - a.x s)
        C, S = f"R({lit(c)})", f"R({lit(s)})"
        return self.assign(f"{a}.x * {C} + {a}.y * {S}", f"{a}.y * {C} - {a}.x * {S}")

    def dft(self, xs):
        n = len(xs)
        if n == 1:
            return list(xs)
        if n == 2:
            return [self.add(xs[0], xs[1]), self.sub(xs[0], xs[1])]
        p = min(d for d in range(2, n + 1) if n % d == 0)
        if p == n:
            return self.dft_prime(xs)
        q = n // p
        # decimation in time: x[p*m + r]  ->  q-point DFTs, twiddle, p-point DFTs
        subs = [self.dft([xs[p * m + r] for m in range(q)]) for r in range(p)]
        out = [None] * n
        for k in range(q):
            col = [self.twiddle(subs[r][k], Fraction(r * k, n)) for r in range(p)]
            res = self.dft(col)
            for s_ in range(p):
                out[k + q * s_] = res[s_]
        return out

    def dft_prime(self, xs):
        """Symmetric-pair formulation for an odd prime length."""
        n = len(xs)
        h = (n - 1) // 2
        tp = [self.add(xs[k], xs[n - k]) for k in range(1, h + 1)]
        tm = [self.sub(xs[k], xs[n - k]) for k in range(1, h + 1)]
        acc = xs[0]
        for t in tp:
            acc = self.add(acc, t)
        out = [None] * n
        out[0] = acc
        for j in range(1, h + 1):
            rx, ry = [f"{xs[0]}.x"], [f"{xs[0]}.y"]
            sx, sy = [], []
            for k in range(1, h + 1):
                c, s = _cos_sin(Fraction(j * k, n))
                C, S = f"R({lit(c)})", f"R({lit(s)})"
                rx.append(f"{C} * {tp[k - 1]}.x")
                ry.append(f"{C} * {tp[k - 1]}.y")
                sx.append(f"{S} * {tm[k - 1]}.x")
                sy.append(f"{S} * {tm[k - 1]}.y")
            re = self.assign(" + ".join(rx), " + ".join(ry))
            im = self.assign(" + ".join(sx), " + ".join(sy))
            # X_j = re - i*im, X_{n-j} = re + i*im   (forward, w = exp(-2 pi i/n))
            out[j] = self.assign(f"{re}.x + {im}.y", f"{re}.y - {im}.x")
            out[n - j] = self.assign(f"{re}.x - {im}.y", f"{re}.y + {im}.x")
        return out


def gen(r: int) -> str:
    e = Emitter()
    xs = [f"a{i}" for i in range(r)]
    outs = e.dft(xs)
    head = [f"// DFT_{r}, forward (w = exp(-2*pi*i/{r})), in place on a[0..{r - 1}]",
            "template <typename V>",
            f"__device__ __forceinline__ void dft{r}(V (&a)[{r}]) {{",
            "    typedef typename real_of<V>::R R;"]
    head += [f"    const V a{i} = a[{i}];" for i in range(r)]
    tail = [f"    a[{i}] = {o};" for i, o in enumerate(outs)]
    return "\n".join(head + e.lines + tail + ["}", ""])


def main():
    out = [
        "// GENERATED by gen_codelets.py -- do not edit by hand.",
        "// Straight-line DFT butterflies for radices " + ", ".join(map(str, RADICES)) + ".",
        "#pragma once",
        "#include <type_traits>",
        "",
        "template <typename V> struct real_of;",
        "template <> struct real_of<double2> { typedef double R; };",
        "template <> struct real_of<float2> { typedef float R; };",
        "template <typename V> __device__ __forceinline__ V mk(typename real_of<V>::R x, "
        "typename real_of<V>::R y);",
        "template <> __device__ __forceinline__ double2 mk<double2>(double x, double y) "
        "{ return make_double2(x, y); }",
        "template <> __device__ __forceinline__ float2 mk<float2>(float x, float y) "
        "{ return make_float2(x, y); }",
        "",
    ]
    for r in RADICES:
        out.append(gen(r))
    out.append("template <int RADIX, typename V> __device__ __forceinline__ void dft(V (&a)[RADIX]) {")
    for i, r in enumerate(RADICES):
        kw = "if constexpr" if i == 0 else "else if constexpr"
        out.append(f"    {kw} (RADIX == {r}) dft{r}(a);")
    out.append("}")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "codelets.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
