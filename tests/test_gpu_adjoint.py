"""Adjoint of the converged fixed point (mpdpft_adjoint): dL/dV_ext and
dL/dR of the nuclei for L = dvol sum (n - n_target)^2, against central
finite differences of whole FP64 solves (h = 1e-4) and, for mixed
precision, against the FP64 adjoint; wrapped in a torch.autograd.Function
(harness only).

The cluster functional (TF + gradient correction) is run with the Hartree
term and with Dirac exchange separately.  With Hartree the loop converges
to round-off and central differences at h = 1e-4 resolve the gradient to
1e-5.  Dirac exchange gives the density a step at its edge (the
Thomas-Fermi-Dirac discontinuity): the fixed point is not unique there, and
~170 edge points of a 32^3 solve land on the other branch between the +h
and -h solves whatever h is, and which ones do depends on round-off (the
order of the grid sums); differences at h = 1e-3 average over those flips
and agree with the adjoint to ~1e-3 along a direction with a large
derivative, to several per cent along one with a small derivative (the
flips' share of the difference is the same in absolute terms); smaller h
do not resolve anything.  With both terms the loop stalls near CC ~ 1e-10 for the same
reason."""
import numpy as np
import pytest

from mpdpft_b200 import abi
from mpdpft_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS, EDGE, SITES, SPACING = 32, 16.0, 3, 3.0
TIGHT = dict(sc_criterion=1e-14, max_sc_count=400)


INTER = {"hartree": [abi.INT_HARTREE], "dirac": [abi.INT_DIRAC]}


def problem(prec=abi.FP64, jitter=0.05, pos=None, inter="hartree"):
    tight = dict(TIGHT)
    if prec == abi.MIXED:
        tight["sc_criterion"] = 1e-9  # FP32 fields: the loop's round-off floor
    p, vext, v0, nuc = W.cluster_adjoint(steps=STEPS, edge=EDGE, sites=SITES, spacing=SPACING, jitter=jitter,
                                         precision=prec, interactions=INTER[inter], **tight)
    if pos is not None:
        nuc["pos"] = pos
        vext = [W.nuclei_potential(STEPS, EDGE, pos, 3.0, nuc["sigma"])]
    return p, vext, v0, nuc


def solve(eng, p, vext, v0):
    e = eng.Engine(p)
    e.sc_run(vext, v0, check=False)
    return e, e.field(abi.FIELD_DENSITY, 0)


@pytest.fixture(scope="module")
def targets(eng):
    out = {}
    for inter in INTER:
        p, vext, v0, _ = problem(jitter=0.0, inter=inter)
        e, n = solve(eng, p, vext, v0)
        e.close()
        out[inter] = n
    return out


def loss_and_grad(n, nt, dvol):
    return dvol * float(((n - nt) ** 2).sum()), 2.0 * dvol * (n - nt)


def bump(center, width=1.5):
    x = W.axis(STEPS, EDGE)
    X, Y, Z = np.meshgrid(x - center[0], x - center[1], x - center[2], indexing="ij")
    return np.exp(-(X * X + Y * Y + Z * Z) / (2 * width * width)).reshape(-1)


# (interaction, difference step, relative tolerance)
FD_CASES = [("hartree", 1e-4, 1e-5), ("dirac", 1e-3, 1e-1)]


@pytest.mark.parametrize("inter,h,tol", FD_CASES)
def test_adjoint_vext_directional_fd(eng, targets, inter, h, tol):
    target = targets[inter]
    p, vext, v0, _ = problem(inter=inter)
    dvol = (EDGE / STEPS) ** 3
    e, n = solve(eng, p, vext, v0)
    L0, g = loss_and_grad(n, target, dvol)
    grad, it, res, st = e.adjoint(g)
    e.close()
    for c in [(0.5, -0.3, 0.2), (2.0, 1.0, -1.0)]:
        phi = bump(c)
        lp = []
        for sgn in (1, -1):
            e2, n2 = solve(eng, p, [vext[0] + sgn * h * phi], v0)
            e2.close()
            lp.append(loss_and_grad(n2, target, dvol)[0])
        fd = (lp[0] - lp[1]) / (2 * h)
        ad = float(grad @ phi)
        print("%s: V_ext direction %s: adjoint %.9e  FD %.9e  rel %.2e  (adjoint iters %d res %.1e)" %
              (inter, c, ad, fd, abs(ad - fd) / abs(fd), it, res))
        assert abs(ad - fd) <= tol * abs(fd)


@pytest.mark.parametrize("inter,h,tol", FD_CASES)
def test_adjoint_nuclei_fd(eng, targets, inter, h, tol):
    target = targets[inter]
    p, vext, v0, nuc = problem(inter=inter)
    dvol = (EDGE / STEPS) ** 3
    e, n = solve(eng, p, vext, v0)
    L0, g = loss_and_grad(n, target, dvol)
    grad, it, res, st = e.adjoint(g)
    dR = e.adjoint_nuclei(grad, nuc["z"], nuc["pos"], nuc["sigma"])
    e.close()
    for a, k in [(0, 0), (1, 2), (2, 1)]:
        lp = []
        for sgn in (1, -1):
            pos = nuc["pos"].copy()
            pos[a, k] += sgn * h
            p2, vext2, _, _ = problem(pos=pos, inter=inter)
            e2, n2 = solve(eng, p2, vext2, v0)
            e2.close()
            lp.append(loss_and_grad(n2, target, dvol)[0])
        fd = (lp[0] - lp[1]) / (2 * h)
        print("%s: nucleus %d coordinate %d: adjoint %.9e  FD %.9e  rel %.2e" %
              (inter, a, k, dR[a, k], fd, abs(dR[a, k] - fd) / abs(fd)))
        # relative to the coordinate's own derivative, or a tenth of the
        # largest one where the coordinate's is small (the centre nucleus)
        assert abs(dR[a, k] - fd) <= tol * max(abs(fd), 0.1 * np.abs(dR).max())


def test_adjoint_mixed_vs_fp64(eng, targets):
    target = targets["hartree"]
    dvol = (EDGE / STEPS) ** 3
    grads = {}
    for prec in (abi.FP64, abi.MIXED):
        p, vext, v0, _ = problem(prec=prec)
        e, n = solve(eng, p, vext, v0)
        _, g = loss_and_grad(n, target, dvol)
        grads[prec], it, res, st = e.adjoint(g, tol=1e-6 if prec == abi.MIXED else 1e-10, check=False)
        e.close()
        print("prec %d: adjoint iterations %d residual %.1e" % (prec, it, res))
        assert res < (1e-5 if prec == abi.MIXED else 1e-9)
    d = np.abs(grads[abi.MIXED] - grads[abi.FP64]).max() / np.abs(grads[abi.FP64]).max()
    print("mixed vs FP64 adjoint: max |diff| / max |grad| = %.2e" % d)
    assert d < 1e-3


def test_adjoint_autograd(eng, targets):
    """dL/dV_ext through a torch.autograd.Function whose backward calls the
    adjoint: the same gradient as the direct call."""
    torch = pytest.importorskip("torch")
    target = targets["hartree"]
    dvol = (EDGE / STEPS) ** 3
    p, vext, v0, _ = problem()

    class Solve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, v):
            e, n = solve(eng, p, [v.detach().numpy()], v0)
            ctx.engine = e
            return torch.from_numpy(n)

        @staticmethod
        def backward(ctx, grad_n):
            g, it, res, st = ctx.engine.adjoint(grad_n.detach().numpy())
            ctx.engine.close()
            return torch.from_numpy(g)

    v = torch.tensor(vext[0], dtype=torch.float64, requires_grad=True)
    n = Solve.apply(v)
    L = dvol * ((n - torch.from_numpy(target)) ** 2).sum()
    L.backward()
    e, n2 = solve(eng, p, vext, v0)
    _, g = loss_and_grad(n2, target, dvol)
    ref, _, _, _ = e.adjoint(g)
    e.close()
    d = np.abs(v.grad.numpy() - ref).max() / np.abs(ref).max()
    assert d < 1e-9


def test_adjoint_cluster_192_hartree_against_fd(eng):
    """The adjoint at the cluster configuration's size (192^3, 13 Z = 3
    nuclei on [-16, 16]^3) with the Hartree functional: the adjoint system
    converges (residual < 1e-9 in FP64) and dL/dR matches central
    differences of whole FP64 solves (h = 1e-4) to 1e-3 of the largest
    component (measured 3.6e-5 .. 2.3e-4).  With Dirac exchange added (the
    configuration's full functional) the loop's fixed point is not unique at
    the TF-Dirac edge and the adjoint system does not converge (residual
    ~1e-2 after 300 iterations), which is why this check runs without it."""
    pt, vt, v0t, _ = W.cluster_adjoint(precision=abi.FP64, jitter=0.0, interactions=[abi.INT_HARTREE])
    with eng.Engine(pt) as et:
        et.sc_run(vt, v0t)
        nt = et.field(abi.FIELD_DENSITY, 0)
    p, vext, v0, nuc = W.cluster_adjoint(precision=abi.FP64, interactions=[abi.INT_HARTREE])
    dvol = (p.edge / p.steps) ** 3
    with eng.Engine(p) as e:
        e.sc_run(vext, v0)
        n = e.field(abi.FIELD_DENSITY, 0)
        grad, it, res, st = e.adjoint(2.0 * dvol * (n - nt), max_iter=300)
        dR = e.adjoint_nuclei(grad, nuc["z"], nuc["pos"], nuc["sigma"])
    print("192^3 cluster (Hartree): adjoint iterations %d, residual %.1e" % (it, res))
    assert res < 1e-9
    h = 1e-4
    for a, k in [(3, 1), (12, 0)]:
        lp = []
        for sgn in (1, -1):
            pos = nuc["pos"].copy()
            pos[a, k] += sgn * h
            v2 = W.nuclei_potential(p.steps, p.edge, pos, 3.0, nuc["sigma"])
            with eng.Engine(p) as e2:
                e2.sc_run([v2], v0)
                n2 = e2.field(abi.FIELD_DENSITY, 0)
            lp.append(dvol * float(((n2 - nt) ** 2).sum()))
        fd = (lp[0] - lp[1]) / (2 * h)
        print("nucleus %d coordinate %d: adjoint %.8e FD %.8e" % (a, k, dR[a, k], fd))
        assert abs(dR[a, k] - fd) <= 1e-3 * np.abs(dR).max()
