"""Oracle fixtures of three configurations (test infrastructure).

Runs the FP64 CPU oracle (oracle/, OpenMP) once to convergence on
  argon_atom at 128^3 (the headline atom)     -> config_argon_atom_128.npz
  cluster_adjoint at 192^3 (13 Z = 3 nuclei)  -> config_cluster_adjoint_192.npz
  electron_hole at 256^3 (two charged species) -> config_electron_hole_256.npz
to the workloads' SC criterion (CC < 1e-8 three times) and stores what the
GPU parity tests compare against: the total energy, mu
and N per species, the iteration count, the final CC and potential
residual, and the density and potential summed over 16^3 coarse blocks
(oracle.block_sums; density sums times dvol, potential block means).
The full fields (64-270 MB) are not kept.

Usage: python tests/golden/make_config_fixtures.py [argon|cluster|electron_hole|all]
(tens of minutes on 8 cores).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mpdpft_b200 import abi  # noqa: E402
from mpdpft_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

BLOCKS = 16


def save(name, p, res, log, dens, pot, seconds):
    dvol = (p.edge / p.steps) ** p.dim
    S = p.species
    out = dict(
        e_total=res.e_total, iterations=res.iterations, converged=res.converged, cc=res.cc,
        v_residual=res.v_residual,
        mu=np.array([res.mu[s] for s in range(S)]),
        abundance=np.array([res.abundance[s] for s in range(S)]),
        dens_blocks=np.stack([O.block_sums(dens[s], p.steps, p.dim, BLOCKS) * dvol for s in range(S)]),
        pot_blocks=np.stack([O.block_sums(pot[s], p.steps, p.dim, BLOCKS) / (p.steps // BLOCKS) ** p.dim
                             for s in range(S)]),
        cc_log=np.array([l.cc for l in log]),
        oracle_seconds=seconds, oracle_threads=O.num_threads(),
    )
    path = os.path.join(HERE, "config_%s.npz" % name)
    np.savez_compressed(path, **out)
    print("%s: iterations %d converged %d E %.12g mu %s (%.0f s on %d threads) -> %s" %
          (name, res.iterations, res.converged, res.e_total, out["mu"], seconds, O.num_threads(), path), flush=True)


def run(name, p, vext, v0):
    t = time.time()
    res, log, dens, pot = O.sc_run(p, vext, v0)
    save(name, p, res, log, dens, pot, time.time() - t)


def main(which):
    if which in ("argon", "all"):
        p, vext, v0 = W.argon_atom(steps=128, precision=abi.FP64, sc_criterion=1e-8)
        run("argon_atom_128", p, vext, v0)
    if which in ("electron_hole", "all"):
        p, vext, v0 = W.electron_hole(steps=256, precision=abi.FP64, sc_criterion=1e-8)
        run("electron_hole_256", p, vext, v0)
    if which in ("cluster", "all"):
        p, vext, v0, _ = W.cluster_adjoint(steps=192, precision=abi.FP64, sc_criterion=1e-8)
        run("cluster_adjoint_192", p, vext, v0)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "all")
