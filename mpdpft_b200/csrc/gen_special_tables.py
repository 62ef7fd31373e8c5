"""Generate special_tables.inc: Chebyshev tables of the special functions of
the reference's finite-temperature gradient-corrected density (DensityExpression
5, mpDPFT.cpp:3363-3453), which the reference takes from spline tables that
are not part of its checkout (TabFunc_PolyLog*) or from a table file
(TabFunc_CurlyA.dat).

  Fermi-Dirac polylogarithms L_s(x) = Li_s(-e^x) for s = 5/2, 3/2, 1/2,
  -1/2, -3/2 (the reference's polylog("5half" .. "m3half", x)):
    x <  -2        alternating series sum_k (-1)^k e^{kx} / k^s (evaluated
                   directly, no table)
    -2 <= x < 60   Chebyshev series of degree 15 on unit intervals
    x >= 60        Sommerfeld expansion
                   -x^s/Gamma(s+1) [1 + sum_k 2 (1 - 2^{1-2k}) zeta(2k)
                   s (s-1) ... (s-2k+1) x^{-2k}] (coefficients tabulated)
  CurlyA(x) = int_x^inf Ai(t) dt (the reference's CurlyA, mpDPFT.h:231-237):
    Chebyshev series of degree 15 on intervals of width 1/4 over
    [-150, 16); the reference's own forms outside (x < -150: its leading
    asymptotic; x >= 16: the leading asymptotic e^{-z}/(2 sqrt(pi) x^{3/4}),
    z = 2/3 x^{3/2}, below 1e-19 there).

Reference values come from mpmath at 30 digits (polylog, and airyai with
derivative=-1 for the integral of Ai from 0).  Every table entry is fitted
at Chebyshev nodes and checked at interval midpoints; the script fails if
any check exceeds 2e-16 in absolute terms (or relative for |f| > 1).

Usage: python mpdpft_b200/csrc/gen_special_tables.py  (about a minute)
"""
import os
import sys

import mpmath
import numpy as np

mpmath.mp.dps = 30
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "special_tables.inc")

FD_ORDERS = [2.5, 1.5, 0.5, -0.5, -1.5]
FD_X0, FD_X1, FD_DEG = -2, 60, 16          # unit intervals [m, m+1), 16 coefficients
FD_ASYM_TERMS = 16
CA_X0, CA_X1, CA_W, CA_DEG = -150.0, 16.0, 0.25, 16


def cheb_fit(f, a, b, deg):
    """Chebyshev coefficients c_0..c_{deg-1} of f on [a, b] from deg
    Chebyshev-Gauss nodes (mp precision), as floats."""
    n = deg
    xs = [mpmath.cos(mpmath.pi * (k + mpmath.mpf(1) / 2) / n) for k in range(n)]
    fx = [f((b - a) / 2 * x + (a + b) / 2) for x in xs]
    c = []
    for j in range(n):
        s = mpmath.fsum(fx[k] * mpmath.cos(mpmath.pi * j * (k + mpmath.mpf(1) / 2) / n) for k in range(n))
        c.append(float(2 * s / n) * (0.5 if j == 0 else 1.0))
    return c


def cheb_eval(c, a, b, x):
    t = (2 * x - a - b) / (b - a)
    b1 = b2 = 0.0
    for cj in reversed(c[1:]):
        b1, b2 = 2 * t * b1 - b2 + cj, b1
    return t * b1 - b2 + c[0]


def polylog_fd(s, x):
    return mpmath.re(mpmath.polylog(s, -mpmath.exp(x)))


def curly_a(x):
    # int_x^inf Ai = 1/3 - int_0^x Ai
    return mpmath.mpf(1) / 3 - mpmath.airyai(x, derivative=-1)


def check(name, f, c, a, b):
    worst = 0.0
    for x in np.linspace(a, b, 7)[1:-1]:
        ref = f(mpmath.mpf(x))
        got = cheb_eval(c, a, b, x)
        err = abs(got - float(ref)) / max(1.0, abs(float(ref)))
        worst = max(worst, err)
    if worst > 2e-16 * 8:
        sys.exit("%s on [%g, %g): fit error %.2e" % (name, a, b, worst))
    return worst


def fd_asymptotic(s):
    """Coefficients t_k of -x^s/Gamma(s+1) sum_k t_k x^{-2k}."""
    out = [1.0]
    for k in range(1, FD_ASYM_TERMS):
        fall = mpmath.mpf(1)
        for i in range(2 * k):
            fall *= (s - i)
        out.append(float(2 * (1 - mpmath.mpf(2) ** (1 - 2 * k)) * mpmath.zeta(2 * k) * fall))
    return out


def main():
    lines = ["// Generated by gen_special_tables.py (mpmath %s, 30 digits); do not edit." % mpmath.__version__]
    worst = 0.0
    nfd = FD_X1 - FD_X0
    lines.append("// Fermi-Dirac polylogarithms Li_s(-e^x), s = 5/2, 3/2, 1/2, -1/2, -3/2:")
    lines.append("// Chebyshev coefficients on [m, m + 1), m = %d .. %d, %d per interval" % (FD_X0, FD_X1 - 1, FD_DEG))
    lines.append("#define MPDPFT_FD_X0 %d" % FD_X0)
    lines.append("#define MPDPFT_FD_X1 %d" % FD_X1)
    lines.append("#define MPDPFT_FD_DEG %d" % FD_DEG)
    lines.append("#define MPDPFT_FD_ASYM %d" % FD_ASYM_TERMS)
    lines.append("#define MPDPFT_FD_TABLE {\\")
    for s in FD_ORDERS:
        for m in range(FD_X0, FD_X1):
            c = cheb_fit(lambda x: polylog_fd(s, x), m, m + 1, FD_DEG)
            worst = max(worst, check("Li_%g" % s, lambda x: polylog_fd(s, x), c, m, m + 1))
            lines.append("  " + ", ".join("%.17e" % v for v in c) + ",\\")
    lines.append("}")
    lines.append("#define MPDPFT_FD_ASYM_TABLE {\\")
    for s in FD_ORDERS:
        lines.append("  " + ", ".join("%.17e" % v for v in fd_asymptotic(s)) + ",\\")
    lines.append("}")
    lines.append("// 1/Gamma(s + 1) for the same orders")
    lines.append("#define MPDPFT_FD_RGAMMA {" + ", ".join("%.17e" % float(1 / mpmath.gamma(s + 1)) for s in FD_ORDERS) + "}")
    nca = int(round((CA_X1 - CA_X0) / CA_W))
    lines.append("// CurlyA(x) = int_x^inf Ai(t) dt: Chebyshev coefficients on [%g + %g i, + %g), i = 0 .. %d"
                 % (CA_X0, CA_W, CA_W, nca - 1))
    lines.append("#define MPDPFT_CA_X0 (%.1f)" % CA_X0)
    lines.append("#define MPDPFT_CA_X1 (%.1f)" % CA_X1)
    lines.append("#define MPDPFT_CA_W (%.2f)" % CA_W)
    lines.append("#define MPDPFT_CA_N %d" % nca)
    lines.append("#define MPDPFT_CA_DEG %d" % CA_DEG)
    lines.append("#define MPDPFT_CA_TABLE {\\")
    for i in range(nca):
        a = CA_X0 + CA_W * i
        c = cheb_fit(curly_a, a, a + CA_W, CA_DEG)
        worst = max(worst, check("CurlyA", curly_a, c, a, a + CA_W))
        lines.append("  " + ", ".join("%.17e" % v for v in c) + ",\\")
    lines.append("}")
    with open(OUT, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote %s (worst fit error %.2e)" % (OUT, worst))


if __name__ == "__main__":
    main()
