"""Prints the two coefficient tables of det_erf in detmath.h.

Both are Chebyshev interpolants, computed with mpmath at 60 digits on the
Chebyshev nodes of [-1, 1] and written as monomial coefficients in the scaled
variable w (|w| <= 1), each rounded once to the nearest double:

* DBGZ_ERF_SMALL_TABLE: erf(x)/x as a degree-20 polynomial in w = 0.32 x^2 - 1
  on x^2 in [0, 6.25] (|x| < 2.5); interpolation error below 1.5e-18 relative.
* DBGZ_ERFC_MID_TABLE: erfc(x) as a degree-28 polynomial in w = x/1.75 - 17/7
  on x in [2.5, 6]; interpolation error below 1.7e-18 absolute.

Run: python dbgenzpaper_b200/csrc/detmath_fit.py
"""
import mpmath as mp

mp.mp.dps = 60


def chebyshev_monomial(f, lo, hi, deg):
    c, s, n = (lo + hi) / 2, 2 / (hi - lo), deg + 1
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n) for k in range(n)]
    vand = mp.matrix([[w ** j for j in range(n)] for w in nodes])
    return mp.lu_solve(vand, mp.matrix([f(c + w / s) for w in nodes])), c, s


def table(name, coef):
    vals = [float(v).hex() for v in coef]
    rows = [", ".join(vals[i:i + 4]) for i in range(0, len(vals), 4)]
    return "#define %s { \\\n  %s }" % (name, ", \\\n  ".join(rows))


def main():
    small = lambda v: mp.erf(mp.sqrt(v)) / mp.sqrt(v) if v > 0 else 2 / mp.sqrt(mp.pi)
    c1, _, s1 = chebyshev_monomial(small, mp.mpf(0), mp.mpf("6.25"), 20)
    c2, cc2, s2 = chebyshev_monomial(mp.erfc, mp.mpf("2.5"), mp.mpf(6), 28)
    print("/* w = %s * x^2 - 1 */" % float(s1).hex())
    print(table("DBGZ_ERF_SMALL_TABLE", c1))
    print("/* w = %s * x - %s */" % (float(s2).hex(), float(cc2 * s2).hex()))
    print(table("DBGZ_ERFC_MID_TABLE", c2))


if __name__ == "__main__":
    main()
