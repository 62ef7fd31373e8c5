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


def test_airy_against_scipy(oracle_lib):
    """Ai and Ai' of the kinetic energies of the gradient-corrected density
    (gsl_sf_airy_Ai / _Ai_deriv, mpDPFT.cpp:5616, 5666): the negated first
    and second derivatives of the CurlyA Chebyshev series on [-150, 16),
    asymptotic series outside, against scipy."""
    import scipy.special as sp
    # (the second derivative of the series loses more digits: Ai' to 1e-9)
    for lo, hi, tol in [(-150.0, 16.0, 1e-9), (-300.0, -150.0, 1e-10), (16.0, 99.0, 5e-8)]:
        for x in np.linspace(lo, hi, 3001):
            a, b = oracle_lib.airy(x)
            A, Ap, _, _ = sp.airy(x)
            # near a zero of Ai (Ai') the absolute error against the envelope
            env_a = abs(x) ** -0.25 / np.sqrt(np.pi) if x < -1 else abs(A)
            env_b = abs(x) ** 0.25 / np.sqrt(np.pi) if x < -1 else abs(Ap)
            # (values below 1e-15 to 1e-15 tol absolute: the table's own floor)
            assert abs(a - A) <= tol * max(env_a, 1e-15), (x, a, A)
            assert abs(b - Ap) <= tol * max(env_b, 1e-15), (x, b, Ap)


def _cosine_problem(dim, **kw):
    """V = V0 + A cos(2 pi x / L) along the first axis on a small periodic
    grid, with its smoothed Laplacian and |grad V|^2 from the oracle's
    DelField (method 5, the fields the kinetic energies read)."""
    from mpdpft_b200 import workloads as W
    steps, edge = 8, 8.0
    p = abi.make_params(dim=dim, steps=steps, edge=edge, density_expression=abi.DENS_GRADIENT, degeneracy=2.0,
                        abundances=[10.0], interactions=[], smearing_extent=0.5, **kw)
    x = W.axis(steps, edge)
    shape = (steps,) * dim
    xs = x.reshape((steps,) + (1,) * (dim - 1)) * np.ones(shape)
    v = (-1.0 + 1.5 * np.cos(2.0 * np.pi * xs / edge)).reshape(-1)
    return p, v


def test_ekin_ait0_3d_against_scipy(oracle_lib):
    """EkinAiT03D (mpDPFT.cpp:5647-5703) of the oracle's energy against a
    scipy restatement: g/(4 pi^2) int [ (2(mu-V))^{5/2}/5 - lap V (2(mu-V))^{1/2}/6 ]
    where a = |grad V|^{2/3}/2 < Mpp[2], else the Airy average
    int_0^{max(1, 100 - U/a)} Ai(x + U/a) [ (2ax)^{5/2}/5 - lap V (2ax)^{1/2}/6 ] dx
    (U = V - mu) by adaptive quadrature; the oracle doubles its trapezoid
    grid from 64 points up to MaxIteration 4 .. 10 as the reference does."""
    import scipy.integrate as si
    import scipy.special as sp
    p, v = _cosine_problem(3, gradient_form=abi.GRADIENT_FINITE_T, airy_threshold=0.2, internal_acc=1e-12,
                           rel_acc=1e-12)
    mu = 0.3
    g2, lap = oracle_lib.delfield(p, v)
    a = 0.5 * np.cbrt(np.abs(g2))
    assert (a >= 0.2).any() and (a < 0.2).any()
    t = np.empty_like(v)
    for i in range(v.size):
        U, L = v[i] - mu, lap[i]
        if a[i] < 0.2:
            w = -2.0 * U
            t[i] = w ** 2.5 / 5.0 - L * np.sqrt(w) / 6.0 if w > 0 else 0.0
        else:
            x1 = max(1.0, 100.0 - U / a[i])
            f = lambda x: sp.airy(x + U / a[i])[0] * ((2 * a[i] * x) ** 2.5 / 5.0 - L * np.sqrt(2 * a[i] * x) / 6.0)
            t[i] = si.quad(f, 0.0, x1, limit=400, epsabs=0.0, epsrel=1e-11)[0]
    ref = 2.0 / (4.0 * np.pi ** 2) * oracle_lib.integrate(p, t)
    dens = np.full_like(v, 0.1)
    r = oracle_lib.energy(p, [v], [dens], [v], [mu])
    assert abs(r.e_kinetic[0] - ref) <= 1e-7 * abs(ref), (r.e_kinetic[0], ref)
    # with no Airy points the small-gradient integrand everywhere
    p0, _ = _cosine_problem(3, gradient_form=abi.GRADIENT_FINITE_T, airy_threshold=1e300)
    w = np.maximum(-2.0 * (v - mu), 0.0)
    ref0 = 2.0 / (4.0 * np.pi ** 2) * oracle_lib.integrate(p0, w ** 2.5 / 5.0 - lap * np.sqrt(w) / 6.0)
    r0 = oracle_lib.energy(p0, [v], [dens], [v], [mu])
    assert abs(r0.e_kinetic[0] - ref0) <= 1e-13 * abs(ref0)


def test_ekin_2d_against_scipy(oracle_lib):
    """The 2D kinetic energy of DensityExpression 5 (mpDPFT.cpp:5608-5621):
    int g/2 [ lap V CurlyA(y)/(12 pi) - |grad V|^{4/3} (y^2 CurlyA(y) + Ai(y)
    + y Ai'(y))/(8 pi) ] - int V n + mu N, y = 2 (V - mu)/|grad V|^{2/3}
    (Ai = Ai' = 0 from y = 50 on, integrand 0 where |grad V|^2 <= 1e-12),
    with scipy's Airy functions and mpmath's CurlyA = 1/3 - int_0^y Ai."""
    import scipy.special as sp
    p, v = _cosine_problem(2, airy_threshold=1e300)
    mu = 0.3
    g2, lap = oracle_lib.delfield(p, v)
    ab = np.abs(g2)
    t = np.zeros_like(v)
    for i in range(v.size):
        if ab[i] > 1e-12:
            y = 2.0 * (v[i] - mu) / np.cbrt(ab[i])
            ai, aip = sp.airy(y)[:2] if y < 50.0 else (0.0, 0.0)
            ca = mp_curly_a(y)
            t[i] = 1.0 * (lap[i] * ca / (12 * np.pi) - ab[i] ** (2 / 3) * (y * y * ca + ai + y * aip) / (8 * np.pi))
    rng = np.random.default_rng(5)
    dens = rng.uniform(0.0, 0.2, v.size)
    n = oracle_lib.integrate(p, dens)
    ref = oracle_lib.integrate(p, t) - oracle_lib.integrate(p, v * dens) + mu * n
    r = oracle_lib.energy(p, [v], [dens], [v], [mu])
    assert abs(r.e_kinetic[0] - ref) <= 1e-9 * abs(ref), (r.e_kinetic[0], ref)
