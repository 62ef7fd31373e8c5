"""Run a fixed number of SC iterations of a named workload (for profilers).

    python -m mpdpft_b200.run_workload [--workload argon_atom] [--steps 128]
        [--precision mixed|fp64] [--iters 12] [--eager]
    python -m mpdpft_b200.run_workload --workload sweep_2d [--count 256] [--iters 4]

Initialises the solve (sc_init), then issues --iters SC iterations (CUDA
graph replays unless --eager) and synchronises; prints the kernel launches
of one captured iteration.  The convergence test is disabled so that every
iteration does the full work.  sweep_2d runs the batched sweep (mpdpft_batch)
of --count solves at their own grid sizes (or --steps if given) and prints
the wall time of the initialisation and of the iterations.
"""
import time
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from mpdpft_b200 import abi, engine  # noqa: E402
from mpdpft_b200 import workloads as W  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="argon_atom", choices=W.workload_names())
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--iters", type=int, default=12)
    ap.add_argument("--eager", action="store_true")
    a = ap.parse_args()
    prec = abi.MIXED if a.precision == "mixed" else abi.FP64
    if a.workload == "sweep_2d":
        probs = W.sweep_2d(a.count, steps=a.steps, precision=prec, sc_criterion=-1.0, max_sc_count=a.iters + 8)
        with engine.Batch(probs) as b:
            t0 = time.perf_counter()
            b.sc_init()
            t1 = time.perf_counter()
            b.sc_step(a.iters)
            b.sync()
            t2 = time.perf_counter()
        print("sweep_2d %d solves: init %.1f ms, %d iterations %.1f ms (%.2f ms each)" %
              (a.count, 1e3 * (t1 - t0), a.iters, 1e3 * (t2 - t1), 1e3 * (t2 - t1) / max(a.iters, 1)), flush=True)
        return
    make = getattr(W, a.workload)
    kw = {} if a.steps is None else {"steps": a.steps}
    p, vext, v0 = make(precision=prec, sc_criterion=-1.0, max_sc_count=a.iters + 8, **kw)
    with engine.Engine(p) as e:
        e.sc_init(vext, v0)
        for _ in range(a.iters):
            e.sc_step(graph=not a.eager)
        e.sync()
        if not a.eager:
            print("iteration kernels %d %s" % (e.iteration_kernels(), e.stage_launch_counts()), flush=True)


if __name__ == "__main__":
    main()
