#!/usr/bin/env python
"""Benchmark of the SC DPFT loop on B200 (one JSON line on rank 0).

Workload (the headline configuration): neutral atom Z = 18 on 128^3, box
[-10, 10]^3 bohr, Gaussian nucleus (sigma 0.1), TF + gradient-corrected
density (the reference's small-gradient branch in its T -> 0 form; spectral
Laplacian smoothed with width 0.2), Hartree by FFT Poisson, Dirac exchange;
mixed precision (FP32 fields and FFTs, FP64 particle-number integral, mu
search, Pulay Gram/solve and energy), one SC iteration replayed as a CUDA
graph.  A step is one SC iteration.  Inputs are synthetic and seeded
(mpdpft_b200.workloads.argon_atom).  The same replay on an all-FP64 context
is extra.fp64_arm; time-to-converge of both (extra.ttc_*) includes the
initial densities.  roofline: the iteration replayed launch by launch from
its graph (CUDA events per launch), the kernel with the largest share of it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The batched half of the metric (extra.batched_sweep): 256 independent 2D
two-species solves of uneven grid size (64^2 .. 512^2, sweep_2d) solved to
convergence in one batch (mpdpft_batch, one CUDA graph replay per iteration
of all solves), against the same 256 solved one after another through
mpdpft_sc_run; solves/s by wall clock, start potentials resident on the GPU
(and, separately, copied from host arrays).

Under torchrun every rank runs an independent replica of the solve (a single
SC solve does not shard); value = iterations of all ranks / max device time.
`--impl reference` times the CPU oracle (the FP64 restatement of the
reference's loop; the reference itself cannot be built here) on the host
cores, rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SC iter/s + time-to-converge @128³ (mixed vs FP64, same GPU); batched solves/s"
UNIT = "SC iter/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--steps-grid", type=int, default=128)
    ap.add_argument("--no-ttc", action="store_true", help="skip the time-to-converge runs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched sweep")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint run")
    ap.add_argument("--no-eh", action="store_true", help="skip the 256^3 electron-hole solves")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (no MEASURED_PEAKS.json: the profiling recipe's 6.65 TB/s)"


def traffic_from_profiles(stage):
    """DRAM bytes per launch of `stage` from profiles/traffic.txt (lines
    "kernel bytes"; # comments), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split("#", 1)[0].split()
            if len(parts) == 2 and parts[0] == stage:
                return float(parts[1])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "mpdpft_bench_clocks_%d_%d.csv" % (os.getpid(), device))

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def host_cpu():
    """(nproc, CPU model) of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return os.cpu_count(), model


def oracle_atom_rate(steps_grid, iters, threads):
    """SC iterations/s of the oracle on `iters` iterations of the atom (after
    its initial density) with `threads` OpenMP threads (0: all)."""
    from oracle import oracle as O
    from mpdpft_b200 import abi, workloads as W
    O.set_threads(threads)
    p, vext, v0 = W.argon_atom(steps=steps_grid, precision=abi.FP64, max_sc_count=iters - 1, sc_criterion=-1.0)
    res, log, dens, v = O.sc_run(p, vext, v0)
    ms = [l.ms for l in log]
    return 1000.0 * len(ms) / sum(ms), len(ms), O.num_threads()


def cpu_baseline(steps_grid, iters=3):
    """The oracle (FP64 C++ restatement of the reference loop, OpenMP) on
    bounded samples: `iters` SC iterations of the headline atom on all host
    threads (the reported value) and on one thread, and a full C1 solve
    (harmonic_tf at 64^3, FP64) on all threads."""
    from oracle import oracle as O
    from mpdpft_b200 import abi, workloads as W
    nproc, model = host_cpu()
    rate, k, threads = oracle_atom_rate(steps_grid, iters, 0)
    rate1, k1, _ = oracle_atom_rate(steps_grid, 1, 1)
    O.set_threads(0)
    p, vext, v0 = W.harmonic_tf(steps=64, precision=abi.FP64)
    t0 = time.perf_counter()
    res, log, dens, v = O.sc_run(p, vext, v0)
    c1_s = time.perf_counter() - t0
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d SC iterations of the %d^3 atom (after its initial density), FP64 oracle" % (k, steps_grid),
            "host": {"nproc": nproc, "cpu_model": model},
            "one_core": {"value": rate1, "unit": UNIT, "cores": 1,
                         "sample": "%d SC iterations of the %d^3 atom on one thread" % (k1, steps_grid)},
            "c1_harmonic_64": {"ttc_s": c1_s, "iterations": res.iterations, "converged": res.converged,
                               "iter_per_s": res.iterations / c1_s, "cores": threads,
                               "sample": "full C1 solve (harmonic_tf 64^3, CC < 1e-12, r_V <= 1e-8)"}}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    from mpdpft_b200 import abi, workloads as W
    O.lib()
    O.set_threads(0)
    # each step is one SC iteration of the oracle on the same workload; the
    # sample is capped so the run ends within a few minutes
    per_iter = 3.5 * 8.0 / max(1, O.num_threads()) * (args.steps_grid / 128.0) ** 3
    k = max(2, min(args.steps, int(120.0 / per_iter)))
    w = min(args.warmup, 2)
    p, vext, v0 = W.argon_atom(steps=args.steps_grid, precision=abi.FP64, max_sc_count=w + k - 1, sc_criterion=-1.0)
    res, log, dens, v = O.sc_run(p, vext, v0)
    ms = [l.ms for l in log[w:w + k]]
    value = 1000.0 * len(ms) / sum(ms)
    nproc, model = host_cpu()
    sample = "%d timed SC iterations (after %d warm-up) of the %d^3 atom, FP64" % (len(ms), w, args.steps_grid)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(ms), "warmup": w, "ms_per_step": float(np.mean(ms)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "argon_atom", "grid": "%d^3" % args.steps_grid, "precision": "fp64",
                       "implementation": "CPU oracle (C++ restatement of the reference loop, OpenMP)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.num_threads(), "kind": "port", "sample": sample,
                             "host": {"nproc": nproc, "cpu_model": model}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def graph_replay(prec, sg, steps, warmup, device, barrier, stream_of):
    """K SC iterations of the atom replayed from one CUDA graph, timed with
    CUDA events on the engine stream after W warm-up iterations.  Returns
    (ms, kernels per iteration, the engine)."""
    import torch
    from mpdpft_b200 import engine, workloads as W
    total = warmup + steps + 16
    p, vext, v0 = W.argon_atom(steps=sg, precision=prec, sc_criterion=-1.0, max_sc_count=total + 8)
    eng = engine.Engine(p, device=device)
    eng.sc_init(vext, v0)
    stream = stream_of(eng)
    for _ in range(warmup):
        eng.sc_step(graph=True)
    eng.sync()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        eng.sc_step(graph=True)
    e1.record(stream)
    e1.synchronize()
    barrier()
    return e0.elapsed_time(e1), eng.iteration_kernels(), eng


def loop_roofline(eng, ms_per_step, iters=5):
    """Per-kernel device time inside the SC loop: `iters` iterations replayed
    launch by launch from the captured graph (mpdpft_iteration_profile, CUDA
    events on the engine stream), aggregated by kernel.  The dominant kernel
    is the one with the largest share of the iteration; achieved = its
    algorithmic bytes per launch / its mean launch time."""
    per = {}
    total = 0.0
    for _ in range(iters):
        for name, ms, b in eng.iteration_profile():
            d = per.setdefault(name, {"ms": 0.0, "launches": 0, "bytes": 0.0})
            d["ms"] += ms
            d["launches"] += 1
            d["bytes"] += b
            total += ms
    peak, peak_kind = measured_peaks()
    kernels = {}
    for name, d in per.items():
        ms_launch = d["ms"] / d["launches"]
        b_launch = d["bytes"] / d["launches"]
        kernels[name] = {"share": d["ms"] / total, "launches_per_iter": d["launches"] // iters,
                         "ms_per_iter": d["ms"] / iters, "ms_per_launch": ms_launch,
                         "bytes_per_launch": b_launch,
                         "GBps": b_launch / (ms_launch / 1000.0) / 1e9 if ms_launch > 0 else None}
    dom = max((k for k in kernels if k != "memset"), key=lambda k: kernels[k]["share"])
    d = kernels[dom]
    ach = d["GBps"]
    return {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": traffic_from_profiles(dom),
            "bytes_per_launch": d["bytes_per_launch"], "ms_per_launch": d["ms_per_launch"],
            "share_of_iteration": d["share"],
            "iteration_sum_ms": total / iters, "graph_ms_per_step": ms_per_step,
            "method": "iteration replayed launch by launch from its CUDA graph, CUDA events per launch, "
                      "mean of %d iterations; bytes: each launch's own input and output fields once" % iters,
            "kernels": kernels}


def run_ours(args, world, rank, local):
    import torch
    from mpdpft_b200 import abi

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    def stream_of(e):
        return torch.cuda.ExternalStream(e.stream(), device=local)

    def max_over_ranks(ms):
        t = torch.tensor([ms], device="cuda")
        if pg:
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    sg = args.steps_grid
    clocks = ClockSampler(local)
    with clocks:
        ms, launches, eng = graph_replay(abi.MIXED, sg, args.steps, args.warmup, local, barrier, stream_of)
    ms_max = max_over_ranks(ms)
    value = world * args.steps / (ms_max / 1000.0)
    roofline = loop_roofline(eng, ms_max / args.steps)
    eng.close()

    # the all-FP64 arm: the same graph replay on an FP64 context
    ms64, launches64, eng64 = graph_replay(abi.FP64, sg, args.steps, args.warmup, local, barrier, stream_of)
    ms64 = max_over_ranks(ms64)
    roof64 = loop_roofline(eng64, ms64 / args.steps, iters=2)
    eng64.close()
    fp64_arm = {"value": world * args.steps / (ms64 / 1000.0), "unit": UNIT, "ms_per_step": ms64 / args.steps,
                "gpu_launches": launches64 * args.steps, "dominant_kernel": roof64["kernel"],
                "dominant_share": roof64["share_of_iteration"], "dominant_frac": roof64["frac"],
                "speedup_mixed_vs_fp64_per_iteration": ms64 / ms_max}

    extra = {"fp64_arm": fp64_arm}
    if not args.no_ttc:
        extra.update(time_to_converge(sg, local))
    e2e = end_to_end(sg, local, abi.MIXED)
    fp64_arm["e2e"] = end_to_end(sg, local, abi.FP64)
    if not args.no_batch:
        extra["batched_sweep"] = batched_sweep(args.batch_count, local, rank=rank, world=world, pg=pg)
    if not args.no_adjoint:
        extra["adjoint_cluster"] = adjoint_cluster(local)
    if not args.no_eh:
        extra["electron_hole_256"] = electron_hole_256(local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(sg)
        except Exception as ex:  # the oracle is test infrastructure; report, do not fail the bench
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": "failed: %s" % ex}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": {"workload": "argon_atom", "grid": "%d^3" % sg, "box": "[-10,10]^3 bohr", "Z": 18,
                           "functional": "TF + gradient correction: the reference's small-gradient branch, T -> 0 "
                                         "form, no |grad V|^2 term (spectral Laplacian smoothed with width 0.2)",
                           "interactions": "Hartree (FFT Poisson, regularised kernel) + Dirac exchange",
                           "precision": "mixed: FP32 fields/FFTs, FP64 N(mu), mu search, Pulay, energy",
                           "graph": "one SC iteration per CUDA graph replay",
                           "parallelism": "replicas x%d" % world,
                           "l2": "no flush; an iteration touches ~150 MB (L2 126 MB), the 2M-point fields of "
                                 "one kernel partly stay in L2 for the next"},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
                "gpu_launches": launches * args.steps, "extra": extra}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def fixture(name):
    p = os.path.join(ROOT, "tests", "golden", "config_%s.npz" % name)
    return dict(np.load(p)) if os.path.exists(p) else None


def against_fixture(name, p, res, dens, pot):
    """Errors of a converged GPU solve against the oracle fixture of its
    configuration (energy, mu, and the density / potential on 16^3 coarse
    blocks)."""
    fx = fixture(name)
    if fx is None:
        return None
    S, dvol, b = p.species, (p.edge / p.steps) ** p.dim, p.steps // 16

    def blocks(f):
        g = np.asarray(f).reshape((16, b) * p.dim)
        return g.sum(axis=tuple(range(1, 2 * p.dim, 2))).reshape(-1)

    return {"dE_over_E": abs(res.e_total - float(fx["e_total"])) / abs(float(fx["e_total"])),
            "coarse_L1_per_particle": max(float(np.abs(blocks(dens[s]) * dvol - fx["dens_blocks"][s]).sum())
                                          / p.abundances[s] for s in range(S)),
            "coarse_potential_max_err": max(float(np.abs(blocks(pot[s]) / b ** p.dim - fx["pot_blocks"][s]).max())
                                            for s in range(S)),
            "mu_abs_err": max(abs(res.mu[s] - float(fx["mu"][s])) for s in range(S)),
            "oracle_iterations": int(fx["iterations"]), "iterations": res.iterations}


def time_to_converge(sg, device):
    """Full solves through mpdpft_sc_run to the SC criterion (CC < 1e-8 three
    times) in mixed and in all-FP64 precision on the same GPU; wall time of
    the whole solve (mpdpft_sc_run: the initial densities, the SC loop, the
    energies) with V_ext set and V_0 resident on the GPU, as for `value`;
    the same with V_0 copied from a host array (ttc_host_*); errors against
    the FP64 oracle fixture."""
    import torch
    from mpdpft_b200 import abi, engine, workloads as W
    out = {}
    acc = {}
    for name, prec in (("mixed", abi.MIXED), ("fp64", abi.FP64)):
        p, vext, v0 = W.argon_atom(steps=sg, precision=prec)
        dev = torch.tensor(v0[0], dtype=torch.float64, device="cuda:%d" % device)
        torch.cuda.synchronize(device)
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0)  # warm-up solve (graph instantiation, clocks)
            path, ms_plane, ms_pass, how = e.fft_config()
            tiles = e.fft_tiles()
            out["fft_%s" % name] = {"path": "plane" if path else "pass", "ms_plane": ms_plane, "ms_pass": ms_pass,
                                    "axis_lines": tiles[0], "z_rows": tiles[1]}
            best_host = None
            for _ in range(3):
                res, log, st = e.sc_run(None, v0)
                best_host = res.seconds if best_host is None else min(best_host, res.seconds)
            best = None
            for _ in range(3):
                res, log, st = e.sc_run(None, device_v0=[dev.data_ptr()])
                best = res if best is None or res.seconds < best.seconds else best
            res = best
            dens = [e.field(abi.FIELD_DENSITY, 0)]
            pot = [e.field(abi.FIELD_POTENTIAL, 0)]
        out["ttc_%s_s" % name] = res.seconds
        out["ttc_host_%s_s" % name] = best_host
        out["device_loop_%s" % name] = res.device_loop
        out["iters_%s" % name] = res.iterations
        out["converged_%s" % name] = res.converged
        out["energy_%s" % name] = res.e_total
        out["mu_%s" % name] = res.mu[0]
        out["iter_per_s_%s" % name] = res.iterations / res.seconds
        acc[name] = against_fixture("argon_atom_%d" % sg, p, res, dens, pot)
    out["ttc_speedup_mixed_vs_fp64"] = out["ttc_fp64_s"] / out["ttc_mixed_s"]
    out["ttc_host_speedup_mixed_vs_fp64"] = out["ttc_host_fp64_s"] / out["ttc_host_mixed_s"]
    out["ttc_note"] = ("wall time of mpdpft_sc_run, best of 3: initial densities, SC loop and energies; "
                       "V_0 resident on the GPU (ttc_host_*: V_0 copied from a host array)")
    out["accuracy_vs_fp64_oracle"] = acc
    return out


def batched_sweep(count, device, reps=3, rank=0, world=1, pg=None):
    """Solves/s of the batched sweep against the same solves one at a time
    (mpdpft_sc_run per solve, contexts created before the timing).  With
    several ranks every rank solves its shard of the solves
    (workloads.sweep_shard, no exchange) and the time is the maximum over
    ranks."""
    import torch
    from mpdpft_b200 import abi, engine, workloads as W
    idx = W.sweep_shard(count, rank, world)
    probs = W.sweep_2d(count, precision=abi.MIXED, indices=idx)

    def tmax(t):  # wall time of the slowest rank
        if pg is None:
            return t
        x = torch.tensor([t], dtype=torch.float64, device="cuda:%d" % device)
        pg.all_reduce(x, op=pg.ReduceOp.MAX)
        return float(x.item())

    def barrier():
        if pg is not None:
            pg.barrier()

    out = {"count": count, "ranks": world, "solves_this_rank": len(idx),
           "grids": {str(s): sum(1 for i in range(count) if W.sweep_steps(i) == s) for s in W.SWEEP_SIZES},
           "precision": "mixed", "timing": "wall clock per full solve of all (max over ranks), best of %d" % reps}
    dev = [torch.tensor(v, dtype=torch.float64, device="cuda:%d" % device) for _, _, v0 in probs for v in v0]
    torch.cuda.synchronize(device)
    with engine.Batch(probs, device=device) as b:
        b.sc_run(device_v0=[x.data_ptr() for x in dev])  # warm-up: graph instantiation
        best = None
        for _ in range(reps):
            barrier()
            t0 = time.perf_counter()
            res, status = b.sc_run(device_v0=[x.data_ptr() for x in dev])
            dt = tmax(time.perf_counter() - t0)
            best = dt if best is None else min(best, dt)
        best_host = None
        for _ in range(reps):
            barrier()
            t0 = time.perf_counter()
            b.sc_run()
            dt = tmax(time.perf_counter() - t0)
            best_host = dt if best_host is None else min(best_host, dt)
    out["batched_solves_per_s"] = count / best
    out["batched_s"] = best
    out["batched_host_inputs_solves_per_s"] = count / best_host
    def tsum(v):  # over ranks
        if pg is None:
            return v
        x = torch.tensor([float(v)], dtype=torch.float64, device="cuda:%d" % device)
        pg.all_reduce(x, op=pg.ReduceOp.SUM)
        return int(round(x.item()))

    out["converged"] = tsum(sum(r.converged for r in res))
    out["status_ok"] = tsum(sum(1 for st in status if st == abi.OK))
    out["iterations_mean"] = float(np.mean([r.iterations for r in res]))
    out["iterations_max"] = int(max(r.iterations for r in res))
    engines = []
    for p, vext, v0 in probs:
        e = engine.Engine(p, device=device)
        for s in range(p.species):
            e.set_external_potential(s, vext[s])
        engines.append(e)
    S = probs[0][0].species
    engines[0].sc_run(None, device_v0=[x.data_ptr() for x in dev[:S]])  # warm-up
    seq_best, seq_host = None, None
    for _ in range(2):
        barrier()
        t0 = time.perf_counter()
        seq = [e.sc_run(None, device_v0=[x.data_ptr() for x in dev[i * S:(i + 1) * S]])[0]
               for i, e in enumerate(engines)]
        dt = tmax(time.perf_counter() - t0)
        seq_best = dt if seq_best is None else min(seq_best, dt)
    barrier()
    t0 = time.perf_counter()
    for e, (p, vext, v0) in zip(engines, probs):
        e.sc_run(None, v0)
    seq_host = tmax(time.perf_counter() - t0)
    for e in engines:
        e.close()
    out["sequential_solves_per_s"] = count / seq_best
    out["sequential_s"] = seq_best
    out["sequential_host_inputs_solves_per_s"] = count / seq_host
    out["speedup_batched_vs_sequential"] = seq_best / best
    out["speedup_host_inputs"] = seq_host / best_host
    out["max_energy_rel_diff_vs_sequential"] = float(max(abs(a.e_total - c.e_total) / abs(c.e_total)
                                                         for a, c in zip(res, seq)))  # this rank's solves
    return out


def electron_hole_256(device):
    """Two charged species on 256^3 (electron_hole): time-to-converge in
    mixed precision and in FP64 on the same GPU (device time of the solve
    loop from the engine), their energy and density differences."""
    from mpdpft_b200 import abi, engine, workloads as W
    out = {"grid": "256^3", "species": 2}
    dens = {}
    acc = {}
    for name, prec in (("mixed", abi.MIXED), ("fp64", abi.FP64)):
        p, vext, v0 = W.electron_hole(steps=256, precision=prec)
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0)  # warm-up (graph instantiation)
            res, log, st = e.sc_run(vext, v0)
            dens[name] = [e.field(abi.FIELD_DENSITY, s) for s in range(2)]
            pot = [e.field(abi.FIELD_POTENTIAL, s) for s in range(2)]
        acc[name] = against_fixture("electron_hole_256", p, res, dens[name], pot)
        out["ttc_%s_s" % name] = res.seconds
        out["iters_%s" % name] = res.iterations
        out["converged_%s" % name] = res.converged
        out["energy_%s" % name] = res.e_total
    out["ttc_speedup_mixed_vs_fp64"] = out["ttc_fp64_s"] / out["ttc_mixed_s"]
    out["energy_rel_err_mixed_vs_fp64"] = abs(out["energy_mixed"] - out["energy_fp64"]) / abs(out["energy_fp64"])
    dv = (40.0 / 256) ** 3
    out["density_l1_per_particle_mixed_vs_fp64"] = float(max(np.abs(dens["mixed"][s] - dens["fp64"][s]).sum() * dv / 20000.0
                                                             for s in range(2)))
    out["accuracy_vs_fp64_oracle"] = acc
    return out


def adjoint_cluster(device, max_iter=60):
    """The 192^3 icosahedral cluster (13 Z = 3 nuclei): converged mixed and
    FP64 solves, L = dvol sum (n - n_target)^2 against the unjittered
    cluster, dL/dV_ext by the adjoint and dL/dR of the 39 coordinates; wall
    times of the solve and of the adjoint."""
    from mpdpft_b200 import abi, engine, workloads as W
    out = {"grid": "192^3", "nuclei": 13, "adjoint_max_iter": max_iter}
    dR = {}
    acc = {}
    for name, prec in (("mixed", abi.MIXED), ("fp64", abi.FP64)):
        pt, vt, v0t, _ = W.cluster_adjoint(precision=prec, jitter=0.0)
        with engine.Engine(pt, device=device) as et:
            et.sc_run(vt, v0t, check=False)
            nt = et.field(abi.FIELD_DENSITY, 0)
        p, vext, v0, nuc = W.cluster_adjoint(precision=prec)
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0, check=False)  # warm-up (graph)
            t0 = time.perf_counter()
            res, log, st = e.sc_run(vext, v0, check=False)
            t1 = time.perf_counter()
            n = e.field(abi.FIELD_DENSITY, 0)
            acc[name] = against_fixture("cluster_adjoint_192", p, res, [n], [e.field(abi.FIELD_POTENTIAL, 0)])
            dvol = (p.edge / p.steps) ** 3
            g = 2.0 * dvol * (n - nt)
            t2 = time.perf_counter()
            grad, it, resid, ast = e.adjoint(g, max_iter=max_iter, check=False)
            t3 = time.perf_counter()
            dR[name] = e.adjoint_nuclei(grad, nuc["z"], nuc["pos"], nuc["sigma"])
        out["solve_s_%s" % name] = t1 - t0
        out["solve_iters_%s" % name] = res.iterations
        out["adjoint_s_%s" % name] = t3 - t2
        out["adjoint_iters_%s" % name] = it
        out["adjoint_residual_%s" % name] = resid
        out["loss_%s" % name] = float(dvol * ((n - nt) ** 2).sum())
    out["max_abs_dL_dR_fp64"] = float(np.abs(dR["fp64"]).max())
    out["dL_dR_rel_diff_mixed_vs_fp64"] = float(np.abs(dR["mixed"] - dR["fp64"]).max() / np.abs(dR["fp64"]).max())
    out["accuracy_vs_fp64_oracle"] = acc
    out["hartree_only"] = adjoint_cluster_hartree(device, max_iter=300)
    return out


def adjoint_cluster_hartree(device, max_iter=300, h=1e-4, coords=((0, 0), (3, 1), (7, 2), (12, 0))):
    """The same cluster with the Hartree functional (Dirac off: with it the
    fixed point is not unique at the TF-Dirac edge and the adjoint system
    does not converge): adjoint residuals in FP64 and mixed precision,
    dL/dR against central differences of whole FP64 solves (step h) for a
    few coordinates, mixed vs FP64 gradient."""
    from mpdpft_b200 import abi, engine, workloads as W
    out = {"interactions": "Hartree", "fd_step": h}
    dR = {}
    for name, prec in (("fp64", abi.FP64), ("mixed", abi.MIXED)):
        pt, vt, v0t, _ = W.cluster_adjoint(precision=prec, jitter=0.0, interactions=[abi.INT_HARTREE])
        with engine.Engine(pt, device=device) as et:
            et.sc_run(vt, v0t, check=False)
            nt = et.field(abi.FIELD_DENSITY, 0)
        p, vext, v0, nuc = W.cluster_adjoint(precision=prec, interactions=[abi.INT_HARTREE])
        dvol = (p.edge / p.steps) ** 3
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0, check=False)
            n = e.field(abi.FIELD_DENSITY, 0)
            t0 = time.perf_counter()
            grad, it, resid, ast = e.adjoint(2.0 * dvol * (n - nt), max_iter=max_iter,
                                             tol=1e-10 if prec == abi.FP64 else 1e-7, check=False)
            out["adjoint_s_%s" % name] = time.perf_counter() - t0
            dR[name] = e.adjoint_nuclei(grad, nuc["z"], nuc["pos"], nuc["sigma"])
        out["adjoint_iters_%s" % name] = it
        out["adjoint_residual_%s" % name] = resid
        if prec == abi.FP64:
            fd_rows = []
            for a, k in coords:
                lp = []
                for sgn in (1, -1):
                    pos = nuc["pos"].copy()
                    pos[a, k] += sgn * h
                    v2 = W.nuclei_potential(p.steps, p.edge, pos, 3.0, nuc["sigma"])
                    with engine.Engine(p, device=device) as e2:
                        e2.sc_run([v2], v0, check=False)
                        n2 = e2.field(abi.FIELD_DENSITY, 0)
                    lp.append(dvol * float(((n2 - nt) ** 2).sum()))
                fd = (lp[0] - lp[1]) / (2 * h)
                fd_rows.append({"nucleus": a, "coord": k, "adjoint": float(dR[name][a, k]), "fd": fd,
                                "rel": abs(float(dR[name][a, k]) - fd) / abs(fd)})
            out["fd_check_fp64"] = fd_rows
    out["dL_dR_rel_diff_mixed_vs_fp64"] = float(np.abs(dR["mixed"] - dR["fp64"]).max() / np.abs(dR["fp64"]).max())
    return out


def end_to_end(sg, device, prec, solves=2):
    """Full solves through the C ABI with host arrays: V_ext and V_0 copied
    in, the density copied out; iterations / wall time."""
    from mpdpft_b200 import abi, engine, workloads as W
    p, vext, v0 = W.argon_atom(steps=sg, precision=prec)
    dens = np.empty(sg ** 3)  # the caller's output array, reused by every solve
    with engine.Engine(p, device=device) as e:
        e.sc_run(vext, v0)
        e.field(abi.FIELD_DENSITY, 0, out=dens)
        iters = 0
        t0 = time.perf_counter()
        for _ in range(solves):
            res, log, st = e.sc_run(vext, v0)
            e.field(abi.FIELD_DENSITY, 0, out=dens)
            iters += res.iterations
        wall = time.perf_counter() - t0
    n = sg ** 3
    return {"value": iters / wall, "unit": UNIT, "h2d_bytes_per_step": int(2 * 8 * n * solves / iters),
            "d2h_bytes_per_step": int(8 * n * solves / iters), "solves": solves,
            "note": "full solves through mpdpft_sc_run with host buffers (V_ext, V_0 in; density out)"}


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
