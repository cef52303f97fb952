"""Generate twiddles.cuh: cos(2 pi m / N) and sin(2 pi m / N) for the register
DFT sizes as double literals.  The angle is reduced exactly (rational
arithmetic) to the first half-quadrant before calling cos/sin, and the
values at multiples of 30 and 45 degrees are exact, so every constant is
within an ulp and symmetric.  Run from this directory:  python gen_twiddles.py"""
import math
from fractions import Fraction


def cos_sin(m, n):
    f = Fraction(m % n, n) * 4  # angle in quarter turns
    q = int(f)
    r = f - q  # in [0, 1): fraction of a quarter turn
    flip = r > Fraction(1, 2)
    rr = 1 - r if flip else r
    if rr == 0:
        c, s = 1.0, 0.0
    elif rr == Fraction(1, 3):
        c, s = math.sqrt(3.0) / 2.0, 0.5
    elif rr == Fraction(1, 2):
        c = s = math.sqrt(0.5)
    else:
        a = float(rr) * math.pi / 2.0
        c, s = math.cos(a), math.sin(a)
    if flip:
        c, s = s, c
    for _ in range(q):
        c, s = -s, c
    return c + 0.0, s + 0.0

SIZES = [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 15, 16]


def main():
    out = ["// Generated by gen_twiddles.py: roots of unity exp(2 pi i m / N) for the",
           "// register DFT sizes.  Do not edit.",
           "#pragma once", "", "namespace pspw {", "",
           "__host__ __device__ constexpr double tw_cos(int N, int m) {"]
    for n in SIZES:
        vals = ", ".join(repr(cos_sin(m, n)[0]) for m in range(n))
        out.append(f"  if (N == {n}) {{ constexpr double t[{n}] = {{{vals}}}; return t[m % {n}]; }}")
    out += ["  return 0.0;", "}", "",
            "__host__ __device__ constexpr double tw_sin(int N, int m) {"]
    for n in SIZES:
        vals = ", ".join(repr(cos_sin(m, n)[1]) for m in range(n))
        out.append(f"  if (N == {n}) {{ constexpr double t[{n}] = {{{vals}}}; return t[m % {n}]; }}")
    out += ["  return 0.0;", "}", "", "}  // namespace pspw", ""]
    open("twiddles.cuh", "w").write("\n".join(out))


if __name__ == "__main__":
    main()
