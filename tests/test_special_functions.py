"""Known answers of the finite-temperature gradient-corrected density
(DensityExpression 5 in 3D, mpDPFT.cpp:3363-3453): the Fermi-Dirac
polylogarithms Li_s(-e^x) and CurlyA(x) = int_x^inf Ai (the tables the GPU
kernels and the oracle share) against mpmath, CurlyA against the
reference's own table TabFunc_CurlyA.dat (when the checkout is present),
and the oracle's density -- small-gradient branch and Airy-averaged branch
-- against a direct mpmath evaluation of the reference's formulas."""
import os

import mpmath
import numpy as np
import pytest

from mpdpft_b200 import abi

mpmath.mp.dps = 30
CURLY_A_TABLE = "/root/reference/TabFunc_CurlyA.dat"


def mp_li(s, x):
    return float(mpmath.re(mpmath.polylog(s, -mpmath.exp(x))))


def mp_curly_a(x):
    return float(mpmath.mpf(1) / 3 - mpmath.airyai(x, derivative=-1))


@pytest.mark.parametrize("s", [2.5, 1.5, 0.5, -0.5, -1.5])
def test_fermi_dirac_polylogs_match_mpmath(oracle_lib, s):
    rng = np.random.default_rng(int(10 * (s + 3)))
    xs = np.concatenate([[-698.0, -60.0, -2.0000001, -2.0, -1.9999999, 0.0, 59.9999999, 60.0, 60.5, 150.0, 698.0],
                         rng.uniform(-40, 80, 40)])
    for x in xs:
        ref = mp_li(s, x)
        got = oracle_lib.polylog(s, x)
        assert abs(got - ref) <= 1e-14 * max(1.0, abs(ref)), (s, x, got, ref)
    # beyond +-699 the reference's own forms: 0 and the leading term
    assert oracle_lib.polylog(s, -800.0) == 0.0
    lead = -800.0 ** s / float(mpmath.gamma(s + 1))
    assert abs(oracle_lib.polylog(s, 800.0) - lead) <= 1e-14 * abs(lead)


def test_curly_a_matches_mpmath(oracle_lib):
    rng = np.random.default_rng(7)
    for x in np.concatenate([[-149.99, -149.98, -100.0, -8.0, 0.0, 1.0, 15.99, 16.0, 20.0], rng.uniform(-149, 16, 60)]):
        ref = mp_curly_a(x)
        got = oracle_lib.curly_a(x)
        assert abs(got - ref) <= 2e-15, (x, got, ref)
    # the reference's own asymptotic below -149.99 and 1 below -1e50
    y = -200.0
    a = (-y) ** 1.5
    assert oracle_lib.curly_a(y) == pytest.approx(1.0 - np.cos(0.25 * np.pi + 2.0 / 3.0 * a) / np.sqrt(np.pi * a),
                                                  abs=1e-13)  # cos of ~1886: the phase's last bits
    assert oracle_lib.curly_a(-1e51) == 1.0


@pytest.mark.skipif(not os.path.exists(CURLY_A_TABLE), reason="reference checkout not present")
def test_curly_a_matches_the_references_table(oracle_lib):
    """TabFunc_CurlyA.dat: (y, CurlyA(y)) pairs at spacing 0.01 on
    [-150, 100], which the reference splines (mpDPFT.cpp:6700)."""
    v = np.loadtxt(CURLY_A_TABLE).reshape(-1)
    y, f = v[0::2], v[1::2]
    sel = (y >= -149.99) & (y < 16.0)
    got = np.array([oracle_lib.curly_a(t) for t in y[sel]])
    err = np.abs(got - f[sel])
    assert err.max() < 1e-12, err.max()
    assert np.all(np.abs(f[y >= 16.0]) < 1e-18)  # where the engine uses the leading asymptotic


def _mp_small_gradient(T, u, lap, g):
    # beta0 (beta1 Li_{3/2} + beta2 Li_{-1/2}), alpha = 1, as the reference writes it
    tau = mpmath.mpf(1) / T
    b0 = -g / (2 * mpmath.pi) ** 1.5
    b1 = tau ** -1.5
    b2 = -mpmath.mpf(lap) / (12 * mpmath.sqrt(tau))
    a = tau * u
    return float(b0 * (b1 * mpmath.re(mpmath.polylog(1.5, -mpmath.exp(a)))
                       + b2 * mpmath.re(mpmath.polylog(-0.5, -mpmath.exp(a)))))


def _mp_airy(T, u, lap, g2, g):
    """int_{-inf}^{100} pre CurlyA(x) (Li_{1/2} + pre2 Li_{-3/2})(-e^{(u + x ar)/T}) dx."""
    tau = mpmath.mpf(1) / T
    b0 = -g / (2 * mpmath.pi) ** 1.5
    b1 = tau ** -1.5
    b2 = -mpmath.mpf(lap) / (12 * mpmath.sqrt(tau))
    ar = mpmath.mpf(g2) ** (mpmath.mpf(1) / 3) / 2
    pre, pre2 = b0 * ar * tau * b1, b2 / b1

    def f(x):
        z = -mpmath.exp((u + x * ar) / T)
        return pre * (mpmath.mpf(1) / 3 - mpmath.airyai(x, derivative=-1)) * (
            mpmath.re(mpmath.polylog(0.5, z)) + pre2 * mpmath.re(mpmath.polylog(-1.5, z)))

    lo = -(u + 40 * T) / ar - 20  # the Fermi factor is below e^-40 there
    return float(mpmath.quad(f, [lo, -10, -2, 0, 4, 100]))


@pytest.mark.parametrize("T,u,lap", [(0.5, 2.0, 0.3), (2.0, -1.0, -0.5), (0.1, 0.4, 1.2)])
def test_finite_t_small_gradient_point(oracle_lib, T, u, lap):
    p = abi.make_params(dim=3, edge=10.0, density_expression=abi.DENS_GRADIENT, degeneracy=2.0,
                        gradient_form=abi.GRADIENT_FINITE_T, airy_threshold=1e300)
    got = oracle_lib.finite_t_point(p, T, u, lap, 0.7)
    ref = _mp_small_gradient(T, u, lap, 2.0)
    assert abs(got - ref) <= 1e-13 * max(1e-300, abs(ref)), (got, ref)


@pytest.mark.parametrize("T,u,lap,g2", [(0.5, 2.0, 0.3, 0.8), (1.0, 0.5, -0.2, 4.0)])
def test_finite_t_airy_branch_point(oracle_lib, T, u, lap, g2):
    """The reference's adaptive Boole rule converges to the Airy integral as
    its Boole pairs and bisection depth grow: at BP = 8, depth 12 and
    InternalAcc 1e-10 it matches mpmath's quadrature of the same integral to
    1e-8.  At the sample input's Mpp = 1 1 (one Boole pair, one
    bisection: 70 integrand values per interval) the rule is coarse -- tens
    of per cent away here, as the reference's own integration would be."""
    p = abi.make_params(dim=3, edge=10.0, density_expression=abi.DENS_GRADIENT, degeneracy=2.0,
                        gradient_form=abi.GRADIENT_FINITE_T, airy_threshold=0.0, boole_pairs=8,
                        boole_max_iter=12, internal_acc=1e-10, abundances=[1e3])
    ref = _mp_airy(T, u, lap, g2, 2.0)
    got = oracle_lib.finite_t_point(p, T, u, lap, g2)
    assert abs(got - ref) <= 1e-8 * abs(ref), (got, ref)
    coarse = abi.make_params(dim=3, edge=10.0, density_expression=abi.DENS_GRADIENT, degeneracy=2.0,
                             gradient_form=abi.GRADIENT_FINITE_T, airy_threshold=0.0, boole_pairs=1,
                             boole_max_iter=1, internal_acc=0.01, abundances=[1e3])
    assert abs(oracle_lib.finite_t_point(coarse, T, u, lap, g2) - ref) <= 0.5 * abs(ref)


def test_bessel_i0e_against_scipy(oracle_lib):
    """e^{-x} I0(x) of the 2D Hartree compensation term (gsl_sf_bessel_I0
    times EXP(-x), mpDPFT.cpp:2659) against scipy's Cephes implementation,
    over the series range, the switch at x = 30 and the asymptotic range."""
    import scipy.special as sp
    xs = np.concatenate([np.linspace(0.0, 40.0, 801), np.geomspace(1e-8, 1e4, 200)])
    err = max(abs(oracle_lib.i0e(x) - sp.i0e(x)) / sp.i0e(x) for x in xs)
    assert err < 1e-14, err
