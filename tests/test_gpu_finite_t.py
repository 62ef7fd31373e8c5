"""GPU parity of the reference's finite-temperature gradient-corrected density
(DensityExpression 5 in 3D, getDenEnAt mpDPFT.cpp:3363-3453): the
small-gradient Fermi-Dirac branch and the Airy-averaged branch with its
adaptive Boole integration (mpDPFT.cpp:3553-3620), pointwise, in the mu
search and in whole SC solves, against the oracle.  Both sides evaluate the
special functions from the same Chebyshev tables (pinned against mpmath
and the reference's TabFunc_CurlyA.dat in tests/test_special_functions.py);
FP64 agrees to round-off, mixed precision to FP32 storage of V and its
derivatives."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def atom(steps, prec, **over):
    kw = dict(gradient_form=abi.GRADIENT_FINITE_T, temperature=[1.0], max_sc_count=60)
    kw.update(over)
    return W.argon_atom(steps=steps, precision=prec, **kw)


@pytest.mark.parametrize("thr", [1e300, 2.0, 0.0])
@pytest.mark.parametrize("prec,tol", [(abi.FP64, 1e-10), (abi.MIXED, 5e-4)])
def test_finite_t_density(eng, oracle_lib, thr, prec, tol):
    """n[V] at a fixed mu: small-gradient branch everywhere (threshold
    1e300), the Airy branch near the nucleus (2.0) and everywhere (0)."""
    p, vext, v0 = atom(24, prec, airy_threshold=thr)
    pr, _, _ = atom(24, abi.FP64, airy_threshold=thr)
    with eng.Engine(p) as e:
        n, N = e.GetDensity(0, v0[0], -5.0)
    nr, Nr = oracle_lib.density(pr, 0, v0[0], -5.0)
    assert rel(n, nr) < tol
    assert abs(N - Nr) / abs(Nr) < tol


@pytest.mark.parametrize("prec", [abi.FP64, abi.MIXED])
def test_finite_t_mu_search(eng, oracle_lib, prec):
    """mu search on V_0 (the bare nucleus) with the Airy branch near the
    nucleus: N(mu) of this functional steps across N* = 18 (from 16.35 to
    30.30 within 1e-9 of mu = -32.6878668), so the reference's bisection
    ends on its trap test (TrappedQ) and the GPU search closes its bracket
    on the same step and reports MPDPFT_WARN_MU_TRAPPED.  Both end at the
    step; in FP64 the oracle's N at the GPU's mu is the GPU's N."""
    p, vext, v0 = atom(32, prec, airy_threshold=2.0, mu=[-10.0])
    pr, _, _ = atom(32, abi.FP64, airy_threshold=2.0, mu=[-10.0])
    with eng.Engine(p) as e:
        mu, N, passes, n, st = e.EnforceConstraints(0, v0[0], 18.0, -10.0, check=False)
    mu_r, ab_r, dens_r, trials, _ = oracle_lib.mu_search(pr, [v0[0]])
    bits_r = oracle_lib.last_status_bits()
    print("GPU mu %.12f N %.10f passes %d status %d; oracle mu %.12f N %.10f trials %d bits %d" %
          (mu, N, passes, st, mu_r[0], ab_r[0], trials, bits_r))
    assert st == abi.WARN_MU_TRAPPED
    assert bits_r & (1 << abi.WARN_MU_TRAPPED)
    assert abs(mu - mu_r[0]) <= (1e-9 if prec == abi.FP64 else 1e-6) * abs(mu_r[0])
    if prec == abi.FP64:
        _, N_r_at_gpu_mu = oracle_lib.density(pr, 0, v0[0], mu)
        assert abs(N - N_r_at_gpu_mu) <= 1e-10 * abs(N_r_at_gpu_mu)


@pytest.mark.parametrize("thr", [1e300, 2.0])
@pytest.mark.parametrize("prec,n_tol", [(abi.FP64, 1e-8), (abi.MIXED, 1e-5)])
def test_finite_t_sc_solve(eng, oracle_lib, thr, prec, n_tol):
    """The atom at 32^3 and T = 1 hartree converged with the finite-T form
    (Airy branch where |grad V|^{2/3}/2 >= 2, or nowhere) against the
    converged oracle: mu, N and the density."""
    p, vext, v0 = atom(32, prec, airy_threshold=thr)
    pr, _, _ = atom(32, abi.FP64, airy_threshold=thr)
    with eng.Engine(p) as e:
        res, log, st = e.sc_run(vext, v0)
        dens = e.field(abi.FIELD_DENSITY, 0)
    res_r, log_r, dens_r, v_r = oracle_lib.sc_run(pr, vext, v0)
    l1 = np.abs(dens - dens_r[0]).sum() * (p.edge / p.steps) ** 3 / 18.0
    print("finite-T atom 32^3 thr %g prec %d: iterations %d (oracle %d), mu %.10f (%.10f), L1/N %.2e" %
          (thr, prec, res.iterations, res_r.iterations, res.mu[0], res_r.mu[0], l1))
    assert res.converged == 1 and res_r.converged == 1
    assert abs(res.abundance[0] - 18.0) <= 2e-9 * 18.0
    # N(mu) of the Airy-averaged form is flat to the tolerance over a short
    # range of mu (the adaptive quadrature and its lower limit change with
    # mu in steps), so searches that both meet the tolerance end up to ~6e-6
    # apart in mu while their densities agree
    assert abs(res.mu[0] - res_r.mu[0]) <= 2e-5 * abs(res_r.mu[0])
    if thr < 1e100:
        # with the Airy branch the searches end at different points of those
        # flat stretches and the loops take different paths (7 vs 9
        # iterations): FP64 agrees to the stopping band (2.8e-7, as mixed),
        # not to round-off
        n_tol = max(n_tol, 1e-6)
    assert l1 < n_tol


@pytest.mark.parametrize("prec,tol", [(abi.FP64, 1e-10), (abi.MIXED, 1e-4)])
def test_finite_t_kinetic_energy(eng, oracle_lib, prec, tol):
    """EkinAiT03D (mpDPFT.cpp:5647-5703) on the GPU against the oracle on
    the GPU's own converged fields: the Airy-averaged kinetic integrand near
    the nucleus (threshold 2) with its trapezoid doubling and the outer
    MaxIteration 4 .. 10 loop, the small-gradient integrand elsewhere."""
    p, vext, v0 = atom(32, prec, airy_threshold=2.0)
    pr, _, _ = atom(32, abi.FP64, airy_threshold=2.0)
    with eng.Engine(p) as e:
        res, log, st = e.sc_run(vext, v0)
        dens = e.field(abi.FIELD_DENSITY, 0).astype(np.float64)
        v = e.field(abi.FIELD_POTENTIAL, 0).astype(np.float64)
    r = oracle_lib.energy(pr, vext, [dens], [v], [res.mu[0]])
    print("E_kin GPU %.12f oracle %.12f; E_ext %.12f %.12f" % (res.e_kinetic[0], r.e_kinetic[0], res.e_external[0],
                                                              r.e_external[0]))
    assert abs(res.e_kinetic[0] - r.e_kinetic[0]) <= tol * abs(r.e_kinetic[0])
    assert abs(res.e_external[0] - r.e_external[0]) <= tol * abs(r.e_external[0])


def test_finite_t_parameters_are_checked(eng):
    for bad in (dict(boole_pairs=0), dict(boole_pairs=51), dict(boole_max_iter=22), dict(internal_acc=0.0),
                dict(temperature=[0.0])):
        p, _, _ = atom(16, abi.FP64, **bad)
        with pytest.raises(eng.MpdpftError) as ex:
            eng.Engine(p)
        assert ex.value.status == abi.ERR_ARG
    p, _, _ = atom(16, abi.FP64, dim=2)
    with pytest.raises(eng.MpdpftError):
        eng.Engine(p)
