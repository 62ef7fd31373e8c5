#!/usr/bin/env python
"""Benchmark of the SC DPFT loop on B200 (one JSON line on rank 0).

Workload (the headline configuration): neutral atom Z = 18 on 128^3, box
[-10, 10]^3 bohr, Gaussian nucleus (sigma 0.1), TF + gradient-corrected
density (spectral grad V and Laplacian smoothed with width 0.2), Hartree by
FFT Poisson, Dirac exchange; mixed precision (FP32 fields and FFTs, FP64
particle-number integral, mu search, Pulay Gram/solve and energy), one SC
iteration replayed as a CUDA graph.  A step is one SC iteration.  Inputs are
synthetic and seeded (mpdpft_b200.workloads.argon_atom).

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
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(stage)
    return None if v is None else float(v)


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


def cpu_baseline(steps_grid, iters=3):
    """The oracle (FP64 C++ restatement of the reference loop, OpenMP) on a
    bounded sample: `iters` SC iterations of the same workload."""
    from oracle import oracle as O
    from mpdpft_b200 import abi, workloads as W
    p, vext, v0 = W.argon_atom(steps=steps_grid, precision=abi.FP64, max_sc_count=iters - 1, sc_criterion=-1.0)
    res, log, dens, v = O.sc_run(p, vext, v0)
    ms = [l.ms for l in log]
    return {"value": 1000.0 * len(ms) / sum(ms), "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": "%d SC iterations of the %d^3 atom (after its initial density), FP64 oracle" % (len(ms), steps_grid)}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    from mpdpft_b200 import abi, workloads as W
    O.lib()
    # each step is one SC iteration of the oracle on the same workload; the
    # sample is capped so the run ends within a few minutes
    per_iter = 3.5 * 8.0 / max(1, O.num_threads()) * (args.steps_grid / 128.0) ** 3
    k = max(2, min(args.steps, int(120.0 / per_iter)))
    w = min(args.warmup, 2)
    p, vext, v0 = W.argon_atom(steps=args.steps_grid, precision=abi.FP64, max_sc_count=w + k - 1, sc_criterion=-1.0)
    res, log, dens, v = O.sc_run(p, vext, v0)
    ms = [l.ms for l in log[w:w + k]]
    value = 1000.0 * len(ms) / sum(ms)
    sample = "%d timed SC iterations (after %d warm-up) of the %d^3 atom, FP64" % (len(ms), w, args.steps_grid)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(ms), "warmup": w, "ms_per_step": float(np.mean(ms)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "argon_atom", "grid": "%d^3" % args.steps_grid, "precision": "fp64",
                       "implementation": "CPU oracle (C++ restatement of the reference loop, OpenMP)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.num_threads(), "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    from mpdpft_b200 import abi, engine, workloads as W

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

    sg = args.steps_grid
    total_iters = args.warmup + args.steps + 16
    p, vext, v0 = W.argon_atom(steps=sg, precision=abi.MIXED, sc_criterion=-1.0, max_sc_count=total_iters + 8)
    eng = engine.Engine(p, device=local)
    eng.sc_init(vext, v0)
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    clocks = ClockSampler(local)
    with clocks:
        for _ in range(args.warmup):
            eng.sc_step(graph=True)
        eng.sync()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            eng.sc_step(graph=True)
        e1.record(stream)
        e1.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], device="cuda")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1000.0)
    launches = eng.iteration_kernels()

    # roofline of the dominant kernel (share = time per launch x launches per
    # iteration); each kernel timed alone with CUDA events on the engine stream
    per_iter = eng.stage_launch_counts()
    stages = {abi.STAGE_SC_MU: ("sc_mu_kernel", 1),
              abi.STAGE_SC_DENSITY: ("sc_density_kernel", 1),
              abi.STAGE_SC_MIX: ("sc_mix_kernel", 1),
              abi.STAGE_FFT_X: ("k_x_roundtrip", per_iter.get("x", 0))}
    if per_iter.get("y", 0) == 0:  # 3D transforms by x-planes
        stages.update({abi.STAGE_FFT_PLANE_FWD: ("k_plane_fwd", per_iter.get("z_r2c", 0)),
                       abi.STAGE_FFT_PLANE_INV: ("k_plane_inv", per_iter.get("z_c2r", 0))})
    else:
        stages.update({abi.STAGE_FFT_Z_R2C: ("k_z_r2c", per_iter.get("z_r2c", 0)),
                       abi.STAGE_FFT_Y: ("k_axis_c2c", per_iter.get("y", 0)),
                       abi.STAGE_FFT_Z_C2R: ("k_z_c2r", per_iter.get("z_c2r", 0))})
    prof = {}
    for st, (name, cnt) in stages.items():
        mst, b = eng.profile_stage(st, reps=20)
        prof[name] = {"ms": mst, "bytes": b, "per_iter": cnt, "share_ms": mst * cnt}
    dom = max(prof, key=lambda k: prof[k]["share_ms"])
    peak, peak_kind = measured_peaks()
    ach = prof[dom]["bytes"] / (prof[dom]["ms"] / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_source": peak_kind,
                "traffic": traffic_from_profiles(dom), "bytes_per_launch": prof[dom]["bytes"],
                "ms_per_launch": prof[dom]["ms"],
                "stages": {k: {"ms": v["ms"], "GBps": v["bytes"] / (v["ms"] / 1000.0) / 1e9 if v["ms"] > 0 else None,
                               "launches_per_iter": v["per_iter"]} for k, v in prof.items()}}
    eng.close()

    extra = {}
    if not args.no_ttc:
        extra = time_to_converge(sg, local)

    e2e = end_to_end(sg, local)
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
                           "functional": "TF + gradient correction (spectral grad V, Laplacian; smoothing 0.2)",
                           "interactions": "Hartree (FFT Poisson, regularised kernel) + Dirac exchange",
                           "precision": "mixed: FP32 fields/FFTs, FP64 N(mu), mu search, Pulay, energy",
                           "graph": "one SC iteration per CUDA graph replay",
                           "parallelism": "replicas x%d" % world,
                           "l2": "inputs larger than L2: an iteration touches ~180 MB (126 MB L2)"},
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
                "gpu_launches": launches * args.steps, "extra": extra}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def time_to_converge(sg, device):
    """Full solves to the SC criterion (CC < 1e-8 three times) in mixed and
    in all-FP64 precision on the same GPU; device time from the engine."""
    from mpdpft_b200 import abi, engine, workloads as W
    out = {}
    dens = {}
    for name, prec in (("mixed", abi.MIXED), ("fp64", abi.FP64)):
        p, vext, v0 = W.argon_atom(steps=sg, precision=prec)
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0)  # warm-up solve (graph instantiation, clocks)
            res, log, st = e.sc_run(vext, v0)
            dens[name] = e.field(abi.FIELD_DENSITY, 0)
            out["ttc_%s_s" % name] = res.seconds
            out["iters_%s" % name] = res.iterations
            out["converged_%s" % name] = res.converged
            out["energy_%s" % name] = res.e_total
            out["mu_%s" % name] = res.mu[0]
            out["iter_per_s_%s" % name] = res.iterations / res.seconds
    out["ttc_speedup_mixed_vs_fp64"] = out["ttc_fp64_s"] / out["ttc_mixed_s"]
    out["energy_rel_err_mixed_vs_fp64"] = abs(out["energy_mixed"] - out["energy_fp64"]) / abs(out["energy_fp64"])
    dv = (20.0 / sg) ** 3
    out["density_l1_per_particle_mixed_vs_fp64"] = float(np.abs(dens["mixed"] - dens["fp64"]).sum() * dv / 18.0)
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
    for name, prec in (("mixed", abi.MIXED), ("fp64", abi.FP64)):
        p, vext, v0 = W.electron_hole(steps=256, precision=prec)
        with engine.Engine(p, device=device) as e:
            e.sc_run(vext, v0)  # warm-up (graph instantiation)
            res, log, st = e.sc_run(vext, v0)
            dens[name] = [e.field(abi.FIELD_DENSITY, s) for s in range(2)]
        out["ttc_%s_s" % name] = res.seconds
        out["iters_%s" % name] = res.iterations
        out["converged_%s" % name] = res.converged
        out["energy_%s" % name] = res.e_total
    out["ttc_speedup_mixed_vs_fp64"] = out["ttc_fp64_s"] / out["ttc_mixed_s"]
    out["energy_rel_err_mixed_vs_fp64"] = abs(out["energy_mixed"] - out["energy_fp64"]) / abs(out["energy_fp64"])
    dv = (40.0 / 256) ** 3
    out["density_l1_per_particle_mixed_vs_fp64"] = float(max(np.abs(dens["mixed"][s] - dens["fp64"][s]).sum() * dv / 20000.0
                                                             for s in range(2)))
    return out


def adjoint_cluster(device, max_iter=60):
    """The 192^3 icosahedral cluster (13 Z = 3 nuclei): converged mixed and
    FP64 solves, L = dvol sum (n - n_target)^2 against the unjittered
    cluster, dL/dV_ext by the adjoint and dL/dR of the 39 coordinates; wall
    times of the solve and of the adjoint."""
    from mpdpft_b200 import abi, engine, workloads as W
    out = {"grid": "192^3", "nuclei": 13, "adjoint_max_iter": max_iter}
    dR = {}
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
    return out


def end_to_end(sg, device, solves=2):
    """Full solves through the C ABI with host arrays: V_ext and V_0 copied
    in, the density copied out; iterations / wall time."""
    from mpdpft_b200 import abi, engine, workloads as W
    p, vext, v0 = W.argon_atom(steps=sg, precision=abi.MIXED)
    with engine.Engine(p, device=device) as e:
        e.sc_run(vext, v0)
        iters = 0
        t0 = time.perf_counter()
        for _ in range(solves):
            res, log, st = e.sc_run(vext, v0)
            e.field(abi.FIELD_DENSITY, 0)
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
