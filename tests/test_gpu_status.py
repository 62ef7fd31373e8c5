"""GPU tests of the status paths and of the reference-layout boundary.

Device loop limits: the mu search's pass cap and the grid barrier's spin
limit are set from the host (mpdpft_set_limits) so small that the kernel
gives up; it must return MPDPFT_ERR_TIMEOUT (no fault, no hang) and the same
context must then solve correctly with the default limits.  Nothing here
faults or hangs a GPU: a spin limit of 0 makes a waiting block leave at its
first poll.

Reference layout: every operator of the ABI is called exactly as a C++
caller of the reference would call it, with host arrays in the reference's
(s+1)^D storage (duplicate planes filled), and compared with the oracle.
"""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("prec", [abi.FP64, abi.MIXED])
def test_mu_pass_cap_times_out_and_context_recovers(eng, oracle_lib, prec):
    p, vext, _ = W.harmonic_tf(steps=32, interactions=[], precision=prec)
    with eng.Engine(p) as e:
        e.set_limits(mu_max_passes=1)
        mu, N, passes, n, st = e.EnforceConstraints(0, vext[0], 1000.0, p.mu[0], check=False)
        assert st == abi.ERR_TIMEOUT
        assert passes == 1
        assert b"pass cap" in e.lib.mpdpft_last_error()
        e.set_limits()  # defaults
        mu, N, passes, n, st = e.EnforceConstraints(0, vext[0], 1000.0, p.mu[0], check=False)
        assert st == abi.OK
    mu_r, ab_r, dens_r, trials, _ = oracle_lib.mu_search(p, vext)
    assert abs(N - 1000.0) / 2000.0 <= 1e-10 * (1 if prec == abi.FP64 else 10)
    assert abs(mu - mu_r[0]) / abs(mu_r[0]) < (1e-8 if prec == abi.FP64 else 1e-6)


def test_barrier_spin_limit_times_out_and_context_recovers(eng):
    """Spin limit 0: the first block that has to wait at a grid barrier of
    the mu kernel gives up, raises the abort word and every block leaves;
    the host reports MPDPFT_ERR_TIMEOUT.  With the default limit the same
    context then runs a full solve."""
    p, vext, v0 = W.harmonic_tf(steps=32, precision=abi.FP64, potential_tol=1e-8)
    with eng.Engine(p) as e:
        e.set_limits(barrier_spin_limit=0)
        mu, N, passes, n, st = e.EnforceConstraints(0, vext[0], 1000.0, p.mu[0], check=False)
        assert st == abi.ERR_TIMEOUT
        assert b"timed out" in e.lib.mpdpft_last_error()
        with pytest.raises(eng.MpdpftError) as ex:
            e.sc_run(vext, v0)
        assert ex.value.status == abi.ERR_TIMEOUT
        e.set_limits()
        res, log, st = e.sc_run(vext, v0)
        assert st == abi.OK and res.converged == 1
        assert abs(res.abundance[0] - 1000.0) <= 2e-7


def test_trapped_search_damps_the_mixing_weight(eng):
    """A mu search that ends inside its bracket without meeting rel_acc (here
    stopped by a pass cap of 2) is the reference's TrappedQ case
    (EnforceConstraints, mpDPFT.cpp:4690-4703): the iteration's status bits
    carry MPDPFT_WARN_MU_TRAPPED and it mixes with theta * min(1,
    |1 - RelDiff|^30), RelDiff = |N* - N| / |N*| (AdmixDensities,
    mpDPFT.cpp:4926-4934); iterations whose search met the tolerance, or
    found no bracket, mix with theta itself."""
    p, vext, v0 = W.harmonic_tf(steps=32, precision=abi.FP64)
    bit = 1 << abi.WARN_MU_TRAPPED
    with eng.Engine(p) as e:
        e.sc_init(vext, v0)
        e.set_limits(mu_max_passes=2)
        logs = [e.sc_step(graph=True, want_log=True) for _ in range(8)]
    trapped = [L for L in logs if L.status_bits & bit]
    print("trapped iterations %d of %d; RelDiff %s" %
          (len(trapped), len(logs), [abs(1000.0 - L.abundance[0]) / 1000.0 for L in trapped]))
    assert trapped
    for L in logs:
        rd = abs(1000.0 - L.abundance[0]) / 1000.0
        mod = min(1.0, abs(1.0 - rd) ** 30) if (L.status_bits & bit) and rd > 1e-12 else 1.0
        assert abs(L.theta[0] - p.theta[0] * mod) <= 1e-15 * p.theta[0]
    assert any(L.theta[0] < p.theta[0] for L in trapped)


def test_set_limits_rejects_bad_values(eng):
    p, _, _ = W.harmonic_tf(steps=16)
    with eng.Engine(p) as e:
        for bad in (0, 25):
            with pytest.raises(eng.MpdpftError) as ex:
                e.set_limits(mu_max_passes=bad)
            assert ex.value.status == abi.ERR_ARG


# ------------------------------------------------------ reference layout --
def _ref(f, dim):
    return W.to_reference(f, dim)


@pytest.mark.parametrize("prec,tol", [(abi.FP64, 1e-11), (abi.MIXED, 2e-5)])
def test_reference_layout_density_and_integral(eng, oracle_lib, prec, tol):
    s, L = 16, 10.0
    p = abi.make_params(dim=3, steps=s, edge=L, density_expression=abi.DENS_TF, degeneracy=2.0, precision=prec)
    v = 0.5 * W.radius2(3, s, L).reshape(-1)
    with eng.Engine(p) as e:
        n, N = e.GetDensity(0, _ref(v, 3), 4.0, layout=abi.LAYOUT_REFERENCE)
    n_r, N_r = oracle_lib.density(p, 0, v, 4.0)
    assert n.size == (s + 1) ** 3
    assert rel(n, _ref(n_r, 3)) < tol
    assert abs(N - N_r) / N_r < tol


@pytest.mark.parametrize("type_", [abi.INT_CONTACT_SELF, abi.INT_DIRAC, abi.INT_HARTREE])
def test_reference_layout_vint(eng, oracle_lib, type_):
    s, L = 16, 8.0
    p = abi.make_params(dim=3, steps=s, edge=L, species=1, beta=0.3, gamma_h=1.0,
                        interactions=[type_], precision=abi.FP64)
    dens = [np.exp(-W.radius2(3, s, L).reshape(-1) / 2.0)]
    with eng.Engine(p) as e:
        got = e.getVint(type_, 0, [_ref(dens[0], 3)], layout=abi.LAYOUT_REFERENCE)
    assert rel(got, _ref(oracle_lib.vint(p, type_, 0, dens), 3)) < 1e-10


@pytest.mark.parametrize("prec,tol", [(abi.FP64, 1e-9), (abi.MIXED, 5e-4)])
def test_reference_layout_delfield(eng, oracle_lib, prec, tol):
    s, L = 24, 12.0
    p = abi.make_params(dim=3, steps=s, edge=L, density_expression=abi.DENS_GRADIENT, smearing_extent=0.6,
                        regularization_threshold=0.4, precision=prec)
    r2 = W.radius2(3, s, L).reshape(-1)
    f = -3.0 / np.sqrt(r2 + 0.5) + 0.1 * np.exp(-0.2 * r2)
    with eng.Engine(p) as e:
        g2, lap = e.DelField(_ref(f, 3), layout=abi.LAYOUT_REFERENCE)
    g2r, lapr = oracle_lib.delfield(p, f)
    assert rel(lap, _ref(lapr, 3)) < tol
    assert rel(g2, _ref(g2r, 3)) < tol


@pytest.mark.parametrize("prec", [abi.FP64, abi.MIXED])
def test_reference_layout_mu_search(eng, oracle_lib, prec):
    p, vext, _ = W.harmonic_tf(steps=32, interactions=[], precision=prec)
    with eng.Engine(p) as e:
        mu, N, passes, n, st = e.EnforceConstraints(0, _ref(vext[0], 3), 1000.0, p.mu[0],
                                                    layout=abi.LAYOUT_REFERENCE)
        N_ref_layout = e.Integrate(n, layout=abi.LAYOUT_REFERENCE)
    mu_r, ab_r, dens_r, trials, _ = oracle_lib.mu_search(p, vext)
    assert n.size == 33 ** 3
    assert abs(N - 1000.0) / 2000.0 <= 1e-10 * (1 if prec == abi.FP64 else 10)
    assert abs(mu - mu_r[0]) / abs(mu_r[0]) < (1e-8 if prec == abi.FP64 else 1e-6)
    # the refilled duplicate planes make the Riemann sum of the returned
    # reference-layout density the periodic integral
    assert abs(N_ref_layout - N) / N < (1e-12 if prec == abi.FP64 else 1e-6)


def test_reference_layout_admix(eng, oracle_lib):
    s, dim, scope, theta = 8, 3, 4, 0.4
    p = abi.make_params(dim=dim, steps=s, edge=4.0, mixer=1, pulay_scope=scope, theta=[theta],
                        precision=abi.FP64, max_sc_count=100)
    n = s ** dim
    rng = np.random.default_rng(7)
    A = 0.3 * rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    x = rng.standard_normal(n)
    nin, nout = [], []
    with eng.Engine(p) as e:
        for t in range(6):
            nin.append([x.copy()])
            nout.append([A @ x + b])
            outs, coeffs, st = e.AdmixDensities([_ref(x, 3)], [_ref(A @ x + b, 3)], [theta],
                                                layout=abi.LAYOUT_REFERENCE)
            assert outs[0].size == (s + 1) ** 3
            x = W.to_periodic(outs[0], 3)
    ref, ref_coeffs, used = oracle_lib.pulay_sequence(p, nin, nout)
    assert rel(x, ref[-1][0]) < 1e-9
    assert np.allclose(coeffs, ref_coeffs, rtol=1e-8, atol=1e-11)
