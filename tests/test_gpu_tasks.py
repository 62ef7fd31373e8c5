"""GPU tests of the task drivers (mpdpft_b200/tasks.py) and of the batched
2D Coulomb terms they use: TaskType 5 parameter exploration over the trap
prefactor and the Hartree strength as one batch, against the same solves one
at a time and against the oracle; the TaskType 1 mu grid at fixed mu."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import tasks as T

pytestmark = pytest.mark.gpu


def single(eng, problem):
    p, vext, v0 = problem
    with eng.Engine(p) as e:
        res, log, st = e.sc_run(vext, v0)
        return res, e.field(abi.FIELD_DENSITY, 0)


def test_batched_coulomb_2d_matches_single_and_oracle(eng, oracle_lib):
    """Three two-species 2D solves with inter-species contact and 2D Hartree
    terms on two grid sizes, as one batch (the Coulomb transform of each
    species batched per grid size ahead of the V assembly), against each
    solved alone and against the converged oracle, at the batch tests'
    tolerances (the batch sums in another order than a solve alone, so the
    loops stop at the same exit test but not at the same point)."""
    problems = [T.trapped_gas_2d(mpp=0.5, gamma_h=1.0, steps=32), T.trapped_gas_2d(mpp=0.6, gamma_h=0.5, steps=64),
                T.trapped_gas_2d(mpp=0.4, gamma_h=1.5, steps=64)]
    from mpdpft_b200 import engine
    with engine.Batch(problems) as b:
        res, status = b.sc_run()
        dens = [b.field(i, abi.FIELD_DENSITY, 0) for i in range(3)]
    assert all(st == abi.OK for st in status)
    for i, (p, vext, v0) in enumerate(problems):
        r1, n1 = single(eng, problems[i])
        rr, _, dr, _ = oracle_lib.sc_run(p, vext, v0)
        dvol = (p.edge / p.steps) ** 2
        de1 = abs(res[i].e_total - r1.e_total) / abs(r1.e_total)
        de = abs(res[i].e_total - rr.e_total) / abs(rr.e_total)
        l1 = np.abs(dens[i] - dr[0]).sum() * dvol / p.abundances[0]
        print("solve %d (%d^2): iterations %d / alone %d / oracle %d; dE/E vs alone %.1e, vs oracle %.1e, "
              "L1/N vs oracle %.1e" % (i, p.steps, res[i].iterations, r1.iterations, rr.iterations, de1, de, l1))
        assert res[i].converged == 1 and r1.converged == 1 and rr.converged == 1
        assert abs(res[i].iterations - r1.iterations) <= 2
        assert de1 < 1e-6 and de < 1e-6 and l1 < 1e-5


def test_parameter_exploration_type5(eng, tmp_path):
    """TaskType 5 over (mpp, gammaH) on a 2 x 2 grid as one batch: the
    figure of merit against the density of the grid's last point, solved
    alone, is ~0 there and positive elsewhere, and the rows land in the
    exploration file."""
    box = [[0.4, 0.6], [0.5, 1.0]]
    ref_res, ref = single(eng, T.trapped_gas_2d(mpp=0.6, gamma_h=1.0))
    out = tmp_path / "mpDPFT_TASKParameterExploration.dat"
    rows, res, status, how = T.parameter_exploration(5, T.trapped_gas_2d, box, 2, ref, out_path=str(out))
    print("rows", rows, "how", how)
    assert how == "batch"
    assert all(st == abi.OK for st in status)
    assert [r[1:] for r in rows] == [[0.4, 0.5], [0.4, 1.0], [0.6, 0.5], [0.6, 1.0]]
    assert abs(rows[-1][0]) < 1e-10
    assert all(r[0] > 1e-6 for r in rows[:-1])
    lines = out.read_text().strip().splitlines()
    assert len(lines) == 4 and all(len(l.split()) == 3 for l in lines)
    assert float(lines[-1].split()[1]) == 0.6


def test_mu_grid_fixed_mu(eng):
    """TaskType 1 at fixed mu (rel_acc 0: no particle-number constraint, the
    reference's grand-canonical runs): every solve keeps its grid mu, and N
    grows with mu along each axis."""
    builder = lambda **kw: T.trapped_gas_2d(rel_acc=0.0, **kw)
    out = T.mu_grid(builder, 4)
    for o in out:
        print(o)
        assert o["converged"] == 1
        assert o["mu"] == pytest.approx(o["mu_start"], rel=1e-15)
    assert out[0]["how"] == "batch"
    assert out[1]["abundance"][1] > out[0]["abundance"][1]
    assert out[2]["abundance"][0] > out[0]["abundance"][0]
