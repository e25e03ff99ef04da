"""Write twiddles.cuh: cos/sin(2*pi*e/n) for the small FFT radices (n <= 27).

Values are evaluated with 50-digit decimal Taylor series and rounded once to
binary64, so every constant is the correctly rounded value.
Run:  python gen_twiddles.py  (from this directory).
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import os

getcontext().prec = 60


def _pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(x):
        x = Decimal(x)
        s, t, k, x2 = Decimal(0), 1 / x, 0, x * x
        while True:
            term = t / (2 * k + 1)
            if term == 0 or abs(term) < Decimal(10) ** -58:
                break
            s += -term if k % 2 else term
            t /= x2
            k += 1
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


PI = _pi()
NMAX = 27  # the 6D passes use n <= 14; the length-M rank-1 FFT radices go to 27


def _cos_sin(frac):
    a = 2 * PI * Decimal(frac.numerator) / Decimal(frac.denominator)
    c, s = Decimal(0), Decimal(0)
    term = Decimal(1)
    k = 0
    while abs(term) > Decimal(10) ** -58 or k < 4:
        if k % 2 == 0:
            c += term if (k // 2) % 2 == 0 else -term
        else:
            s += term if (k // 2) % 2 == 0 else -term
        k += 1
        term = term * a / k
    snap = lambda v: 0.0 if abs(v) < Decimal(10) ** -40 else float(v)
    return snap(c), snap(s)


def main():
    cases_c, cases_s = [], []
    for n in range(1, NMAX + 1):
        for e in range(n):
            c, s = _cos_sin(Fraction(e, n) % 1)
            cases_c.append(f"    case {n * 32 + e}: return {c!r};")
            cases_s.append(f"    case {n * 32 + e}: return {s!r};")
    out = [
        f"// cos(2*pi*e/n) and sin(2*pi*e/n) for n in [1,{NMAX}], e in [0,n), correctly",
        "// rounded to binary64.  Generated by gen_twiddles.py; do not edit.",
        "#pragma once",
        "namespace fame {",
        "__host__ __device__ constexpr double tw_cos(int n, int e) {",
        "  switch (n * 32 + e) {", *cases_c, "    default: return 0.0;", "  }", "}",
        "__host__ __device__ constexpr double tw_sin(int n, int e) {",
        "  switch (n * 32 + e) {", *cases_s, "    default: return 0.0;", "  }", "}",
        "}  // namespace fame", "",
    ]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "twiddles.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main()
