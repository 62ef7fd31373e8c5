"""Run a fixed number of SC iterations of a named workload (for profilers).

    python -m mpdpft_b200.run_workload [--workload argon_atom] [--steps 128]
        [--precision mixed|fp64] [--iters 12] [--eager]

Initialises the solve (sc_init), then issues --iters SC iterations (CUDA
graph replays unless --eager) and synchronises; prints the kernel launches
of one captured iteration.  The convergence test is disabled so that every
iteration does the full work.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from mpdpft_b200 import abi, engine  # noqa: E402
from mpdpft_b200 import workloads as W  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="argon_atom", choices=W.workload_names())
    ap.add_argument("--steps", type=int, default=128)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--iters", type=int, default=12)
    ap.add_argument("--eager", action="store_true")
    a = ap.parse_args()
    prec = abi.MIXED if a.precision == "mixed" else abi.FP64
    make = getattr(W, a.workload)
    p, vext, v0 = make(steps=a.steps, precision=prec, sc_criterion=-1.0, max_sc_count=a.iters + 8)
    with engine.Engine(p) as e:
        e.sc_init(vext, v0)
        for _ in range(a.iters):
            e.sc_step(graph=not a.eager)
        e.sync()
        if not a.eager:
            print("iteration kernels %d %s" % (e.iteration_kernels(), e.stage_launch_counts()), flush=True)


if __name__ == "__main__":
    main()
