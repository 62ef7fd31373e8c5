"""The reference's outer task loops (mpDPFTmain.cpp:60-160) on the GPU
engine: each task's independent SC solves run together, as one batch
(mpdpft_batch: 2D solves with the gradient-corrected functional) or one
context after another (everything else).

  mu_grid               TaskType 1: the rectangular mu grid of RetrieveTask
                        (mpDPFT.cpp:6071-6078)
  parameter_exploration TaskType 5, 6, 7: the hyperbox grid of the main loop
                        (mpDPFTmain.cpp:110-160) with the parameters
                        RetrieveTask assigns (mpDPFT.cpp:6087-6101) and the
                        figure of merit of GetFigureOfMerit (mpDPFT.cpp:13786-13788),
                        written as mpDPFT_TASKParameterExploration.dat
                        (mpDPFT.cpp:13232-13243)

A problem builder is a callable returning (params, vext list, v0 list), as
the builders in workloads.py do; the drivers pass it the task's parameters
as keyword arguments.
"""
import numpy as np

from . import abi, engine, workloads as W


def mu_grid_points(mu, count):
    """The start mu of each of the `count` solves of TaskType 1 for two
    species: AxesPoints = round(count^(1/2)), solve c scales mu_0 by
    (1 + delta)^p0 and mu_1 by (1 + delta)^p1, p0 = c div AxesPoints,
    p1 = c mod AxesPoints, delta = 1.1^(1/AxesPoints) - 1."""
    if len(mu) != 2:
        raise ValueError("the reference's mu grid is defined for two species")
    if count <= 1:
        return [list(mu)]
    axes = int(round(count ** 0.5))
    delta = 1.1 ** (1.0 / axes) - 1.0
    out = []
    for c in range(count):
        p0, p1 = (c - c % axes) // axes, c % axes
        out.append([mu[0] * (1.0 + delta) ** p0, mu[1] * (1.0 + delta) ** p1])
    return out


# the parameters each task type varies, in the order of task.VEC
TASK_PARAMETERS = {7: ("mpp",), 5: ("mpp", "gamma_h"), 6: ("tau", "mpp", "gamma_h")}


def hyperbox_points(task_type, hyperbox, count):
    """task.VEC of every solve, in the loop order of mpDPFTmain.cpp:114-160:
    axis i runs over hyperbox[i][0] + (hyperbox[i][1] - hyperbox[i][0]) t /
    (count - 1), t = 0 .. count - 1, the first axis outermost."""
    names = TASK_PARAMETERS[task_type]
    if len(hyperbox) < len(names):
        raise ValueError("TaskType %d needs a hyperbox of %d axes" % (task_type, len(names)))
    if count < 2:
        raise ValueError("the parameter exploration needs TaskParameterCount >= 2")
    axes = [[lo + (hi - lo) * t / (count - 1.0) for t in range(count)] for lo, hi in hyperbox[:len(names)]]
    pts = [[]]
    for ax in axes:
        pts = [p + [v] for p in pts for v in ax]
    return pts


def figure_of_merit(p, density, reference):
    """1 - 2 <n, n_ref> / (|n|^2 + |n_ref|^2) of species 0 over the stored
    points of the reference layout (GetFigureOfMerit, mpDPFT.cpp:13786-13788,
    VecMult :7103-7107): duplicate planes count as stored points."""
    a = W.to_reference(np.asarray(density), p.dim)
    b = np.asarray(reference)
    if b.size != a.size:
        b = W.to_reference(b, p.dim)
    return 1.0 - 2.0 * float(a @ b) / (float(a @ a) + float(b @ b))


def _batchable(problems):
    p0 = problems[0][0]
    return all(p.dim == 2 and p.density_expression == abi.DENS_GRADIENT and p.species == p0.species
               and p.precision == p0.precision for p, _, _ in problems)


def solve_all(problems, device=0, want_density=True):
    """Solve every problem; returns (results, statuses, densities of species
    0 or None, how) with how = 'batch' or 'sequential'."""
    if _batchable(problems):
        with engine.Batch(problems, device=device) as b:
            res, status = b.sc_run(check=False)
            dens = [b.field(i, abi.FIELD_DENSITY, 0) for i in range(len(problems))] if want_density else None
        return list(res), list(status), dens, "batch"
    res, status, dens = [], [], []
    for p, vext, v0 in problems:
        with engine.Engine(p, device=device) as e:
            r, log, st = e.sc_run(vext, v0, check=False)
            res.append(r)
            status.append(st)
            if want_density:
                dens.append(e.field(abi.FIELD_DENSITY, 0))
    return res, status, (dens if want_density else None), "sequential"


def mu_grid(builder, count, device=0):
    """TaskType 1: the solves of the mu grid, started from builder()'s mu.
    Returns a list of dicts (mu start, mu, N, E, converged, status)."""
    p, _, _ = builder()
    starts = mu_grid_points(list(p.mu)[:p.species], count)
    problems = [builder(mu=m) for m in starts]
    res, status, _, how = solve_all(problems, device, want_density=False)
    return [dict(mu_start=m, mu=list(r.mu)[:p.species], abundance=list(r.abundance)[:p.species], e_total=r.e_total,
                 converged=r.converged, status=st, how=how) for m, r, st in zip(starts, res, status)]


def parameter_exploration(task_type, builder, hyperbox, count, reference, device=0, out_path=None):
    """TaskType 5, 6 or 7: one solve per point of the hyperbox grid, each
    given the task's parameters (7: mpp; 5: mpp, gamma_h; 6: tau, mpp,
    gamma_h) by keyword; the figure of merit of its species-0 density
    against `reference`.  Returns the rows [FOM, VEC...] of the reference's
    ParameterExplorationContainer and writes them to out_path (16 digits,
    one row a line) when given."""
    names = TASK_PARAMETERS[task_type]
    pts = hyperbox_points(task_type, hyperbox, count)
    problems = [builder(**dict(zip(names, v))) for v in pts]
    res, status, dens, how = solve_all(problems, device)
    rows = []
    for v, (p, _, _), n in zip(pts, problems, dens):
        rows.append([figure_of_merit(p, n, reference)] + list(v))
    if out_path:
        with open(out_path, "w") as f:
            for r in rows:
                f.write(" ".join("%.16g" % x for x in r) + " \n")
    return rows, res, status, how


def trapped_gas_2d(mpp=0.5, gamma_h=1.0, tau=1.0, mu=None, steps=64, edge=16.0, n_target=(20.0, 20.0),
                   precision=abi.FP64, coulomb=True, seed=W.SEED_BASE + 7, **over):
    """A builder for the task drivers: two species in the 2D trap
    V_ext = mpp r^2 (Env 1), the 2D gradient-corrected density at the
    automatic temperature, inter-species contact coupling (type 1) and, with
    coulomb, the 2D Hartree repulsion of each species (type 8, strength
    gamma_h); tau enters the TF-inspired functionals only (the gradient form
    has none).  V_0 = V_ext + U(-1e-3, 1e-3)."""
    ints = [abi.INT_CONTACT_MUTUAL] + ([abi.INT_HARTREE] if coulomb else [])
    mu0 = [float(np.sqrt(4.0 * mpp * n / 2.0 / np.pi)) + 1.0 for n in n_target] if mu is None else list(mu)
    kw = dict(dim=2, steps=steps, species=2, edge=edge, abundances=list(n_target), rel_acc=1e-10,
              density_expression=abi.DENS_GRADIENT, degeneracy=2.0, interactions=ints, beta=0.3, gamma_h=gamma_h,
              mu=mu0, temperature=[-1.0, -1.0], tau=[tau, tau], mixer=1, pulay_scope=6, theta=[0.3, 0.3],
              sc_criterion=1e-10, max_sc_count=300, smearing_extent=1.5 * edge / steps,
              regularization_threshold=0.45, precision=precision)
    kw.update(over)
    p = abi.make_params(**kw)
    vext = (mpp * W.radius2(2, steps, edge)).reshape(-1)
    v0 = [vext + W.noise(vext.shape, 1e-3, seed + 100 * q) for q in range(2)]
    return p, [vext, vext.copy()], v0
