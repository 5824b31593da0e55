"""Generate core/bessel_table.inc: Chebyshev fits of the modified-Bessel ratios K1(x)/K2(x) and K0(x)/K2(x).

The thermal Faraday coefficients need the two ratios at x = 1/Theta_e for 0.2 <= x < 30 (hotter plasma uses the
asymptotic forms, colder the Hankel series).  This script samples the ratios with mpmath at 40 significant digits,
fits each piece [a, b) with a Chebyshev series in
z = (2 ln x - ln a - ln b) / (ln b - ln a), keeps the terms that matter at double precision and writes them as a C
table.  A second, shorter length per piece is recorded for single-precision evaluation (terms below 2^-26 of the
leading one dropped).

usage: python gen_bessel_table.py > ../core/bessel_table.inc
"""
import numpy as np
from numpy.polynomial import chebyshev as Ch
import mpmath

mpmath.mp.dps = 40

PIECES = [(0.2, 0.5), (0.5, 1.2), (1.2, 3.0), (3.0, 7.0), (7.0, 15.0), (15.0, 30.0)]
DEG = 22


def ratios(x):
    x = np.atleast_1d(x)
    r10 = np.empty(x.shape)
    r02 = np.empty(x.shape)
    for i, v in enumerate(x.flat):
        v = mpmath.mpf(float(v))
        k0, k1, k2 = mpmath.besselk(0, v), mpmath.besselk(1, v), mpmath.besselk(2, v)
        r10.flat[i] = float(k1 / k2)
        r02.flat[i] = float(k0 / k2)
    return r10, r02


def fit(a, b):
    la, lb = np.log(a), np.log(b)
    # Chebyshev-Gauss nodes in z, mapped to x
    n = 64
    z = np.cos(np.pi * (np.arange(n) + 0.5) / n)
    x = np.exp(0.5 * (z * (lb - la) + (lb + la)))
    r10, r02 = ratios(x)
    c10 = Ch.chebfit(z, r10, DEG)
    c02 = Ch.chebfit(z, r02, DEG)
    return la, lb, c10, c02


def trim(c, tol):
    keep = len(c)
    while keep > 1 and abs(c[keep - 1]) < tol * abs(c[0]):
        keep -= 1
    return keep


def main():
    rows = []
    worst = 0.0
    for a, b in PIECES:
        la, lb, c10, c02 = fit(a, b)
        n64 = max(trim(c10, 1e-18), trim(c02, 1e-18))
        n32 = max(trim(c10, 2.0 ** -26), trim(c02, 2.0 ** -26))
        # check accuracy on a dense grid
        xs = np.exp(np.linspace(la, lb, 301)[:-1])
        z = (2 * np.log(xs) - la - lb) / (lb - la)
        e10 = np.abs(Ch.chebval(z, c10[:n64]) / ratios(xs)[0] - 1).max()
        e02 = np.abs(Ch.chebval(z, c02[:n64]) / ratios(xs)[1] - 1).max()
        worst = max(worst, e10, e02)
        rows.append((a, b, la, lb, n64, n32, c10, c02))
    print("// Generated by phoenix_b200/csrc/tools/gen_bessel_table.py -- do not edit.")
    print("// Chebyshev fits in z = (2 ln x - ln a - ln b) / (ln b - ln a) of K1/K2 and K0/K2 on [a, b);")
    print("// max relative error of the double-length fit on a dense grid: %.2e" % worst)
    print("#define PHX_BESSEL_NPIECE %d" % len(rows))
    print("#define PHX_BESSEL_NCOEF %d" % (DEG + 1))
    print("#define PHX_BESSEL_DATA \\")
    print("  { \\")
    for a, b, la, lb, n64, n32, c10, c02 in rows:
        print("    {%.17g, %.17g, %.17g, %.17g, %d, %d, \\" % (a, b, la, lb, n64, n32))
        print("     {" + ", ".join("%.17g" % v for v in c10) + "}, \\")
        print("     {" + ", ".join("%.17g" % v for v in c02) + "}}, \\")
    print("  }")


if __name__ == "__main__":
    main()
