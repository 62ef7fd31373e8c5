"""Host logic of the task drivers (mpdpft_b200/tasks.py): the TaskType 1
mu grid (RetrieveTask, mpDPFT.cpp:6071-6078), the hyperbox grids of
TaskType 5/6/7 (mpDPFTmain.cpp:110-160), the figure of merit
(GetFigureOfMerit, mpDPFT.cpp:13786-13788) and the exploration file's
format.  No GPU."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import tasks as T
from mpdpft_b200 import workloads as W


def test_mu_grid_points_follow_retrieve_task():
    mu = [2.0, 3.0]
    pts = T.mu_grid_points(mu, 9)
    axes = 3
    delta = 1.1 ** (1.0 / axes) - 1.0
    assert len(pts) == 9
    for c, (a, b) in enumerate(pts):
        p0, p1 = c // axes, c % axes
        assert a == pytest.approx(2.0 * (1 + delta) ** p0, rel=1e-15)
        assert b == pytest.approx(3.0 * (1 + delta) ** p1, rel=1e-15)
    # the grid spans a factor 1.1^((A-1)/A) per axis
    assert pts[-1][0] / pts[0][0] == pytest.approx(1.1 ** (2.0 / 3.0))
    assert T.mu_grid_points(mu, 1) == [mu]
    with pytest.raises(ValueError):
        T.mu_grid_points([1.0], 4)


@pytest.mark.parametrize("task_type,nax", [(7, 1), (5, 2), (6, 3)])
def test_hyperbox_points_loop_order(task_type, nax):
    box = [[0.0, 1.0], [10.0, 20.0], [-1.0, 1.0]]
    pts = T.hyperbox_points(task_type, box, 3)
    assert len(pts) == 3 ** nax
    assert all(len(p) == nax for p in pts)
    # first axis outermost, endpoints included
    assert pts[0] == [box[i][0] for i in range(nax)]
    assert pts[-1] == [box[i][1] for i in range(nax)]
    if nax > 1:
        assert pts[1][0] == pts[0][0] and pts[1][-1] != pts[0][-1]
    with pytest.raises(ValueError):
        T.hyperbox_points(task_type, box, 1)


def test_figure_of_merit():
    p = abi.make_params(dim=2, steps=16, edge=8.0)
    r2 = W.radius2(2, 16, 8.0).reshape(-1)
    n = np.exp(-r2)
    assert T.figure_of_merit(p, n, n) == pytest.approx(0.0, abs=1e-15)
    assert T.figure_of_merit(p, n, W.to_reference(n, 2)) == pytest.approx(0.0, abs=1e-15)
    fom = T.figure_of_merit(p, n, np.exp(-r2 / 2.0))
    a, b = W.to_reference(n, 2), W.to_reference(np.exp(-r2 / 2.0), 2)
    assert fom == pytest.approx(1.0 - 2.0 * (a @ b) / (a @ a + b @ b), rel=1e-14)
    assert 0.0 < fom < 1.0


def test_builder_parameters():
    p, vext, v0 = T.trapped_gas_2d(mpp=0.7, gamma_h=1.3, steps=16)
    assert p.gamma_h == pytest.approx(1.3)
    r2 = W.radius2(2, 16, p.edge).reshape(-1)
    assert np.allclose(vext[0], 0.7 * r2)
    assert abi.INT_HARTREE in list(p.interactions)[:p.n_interactions]
    assert T._batchable([T.trapped_gas_2d(steps=16), T.trapped_gas_2d(steps=32)])
