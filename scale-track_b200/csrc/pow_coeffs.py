"""Derives the single-precision polynomial coefficients of st_pow0687f (st_pow.h).

    python scale-track_b200/csrc/pow_coeffs.py

x^0.687 is split as (1 + t)^0.687 * 2^(r / 1000) * 2^k with t = m - 1, m in [sqrt(1/2),
sqrt(2)) the reduced mantissa, and 687 e = 1000 k + r (r in [0, 1000)) for the binary
exponent e.  Each factor is a polynomial (degree 8 in t, degree 6 in r) fitted by least
squares on Chebyshev nodes in double precision, written out as float hex literals.  The
header holds the printed literals; this script is how they were obtained.
"""
import numpy as np
from numpy.polynomial import chebyshev as C
from numpy.polynomial import polynomial as Pw


def fit(f, a, b, deg, n=40000):
    k = np.arange(n)
    mid, half = (a + b) / 2, (b - a) / 2
    x = np.cos(np.pi * (k + 0.5) / n) * half + mid
    c = C.chebfit((x - mid) / half, f(x), deg)
    p = Pw.Polynomial(C.cheb2poly(c))
    return p(Pw.Polynomial([-mid / half, 1 / half])).coef


def main():
    a0, b0 = np.sqrt(0.5) - 1, np.sqrt(2) - 1
    cm = fit(lambda t: (1 + t) ** 0.687, a0, b0, 8)
    ce = fit(lambda r: 2.0 ** (r / 1000.0), 0.0, 999.0, 6)
    for name, co in (("t", cm), ("r", ce)):
        lits = []
        for c in co:
            h = float(np.float32(c)).hex()          # e.g. 0x1.5fbe760000000p-1
            mant, ex = h.split("p")
            lits.append(mant.rstrip("0").rstrip(".") + "p" + ex + "f")
        print(name, ", ".join(lits))


if __name__ == "__main__":
    main()
