#!/usr/bin/env python
"""Throughput of the filament Brownian-dynamics step on B200.

Metric: segment-steps/s = bonds x reference steps / second, one reference
step (i_step) being one pair-force evaluation plus one integrator half step
(the reference's step loop, src/simulation.cpp:37-62, advances delta/2).

Workload (default): 20,000 filaments x 10 bonds in a 3D periodic cube of side
200, persistence length 100, WCA eps = sigma = 1, dt = 1e-4, thermal noise on
(synthetic, seeded random insertion).  One bench step = one captured-graph
launch of 20 reference steps (10 midpoint BD steps, pair-list rebuilds
included as they fall due), timed with CUDA events on the context's stream;
L2 is flushed (256 MiB write) before every timed launch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1: one process per GPU under torch.distributed.run, each rank an
independent replica (weak scaling, no data-path collective); the time is the
max over ranks.  --impl reference times the reference's own CPU code
(oracle/_ref, OpenMP over all host cores) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "segment-steps/s, 1 B200: mixed+batched vs FP64 GPU at ≤1e-5 force err"
UNIT = "segment-steps/s"
I_STEPS_PER_STEP = 20
# DRAM bytes (read + write) of one k_integrate launch of the default workload,
# mixed precision, from ncu (cold cache): the mean of a midstep launch
# (21.87 MB) and a full-step launch (39.48 MB), which alternate.
TRAFFIC_K_INTEGRATE_MIXED = 30.67e6
WORKLOAD_DESC = ("B: 20,000 filaments x 10 bonds (200,000 segments, 220,000 sites), 3D periodic "
                 "cube side 200, lp 100, WCA eps=sigma=1, dt 1e-4, noise on")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="B")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many host-driven steps and exit (for ncu)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of --profile-steps")
    return ap.parse_args()


def load_measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None
        self.lines = []
        self.windows = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark(self, t0, t1):
        self.windows.append((t0, t1))

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # Samples inside the timed windows (one 20 ms sample period of slack).
        inside = [l for (t, l) in self.lines
                  if any(a - 0.02 <= t <= b + 0.02 for (a, b) in self.windows)]
        for line in inside:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def replica_seed(rank):
    """Seed of the replica a rank runs (independent systems, one per GPU)."""
    return rank


def reduce_max(value, dist):
    """Max over ranks (the device times of all replicas); dist may be None."""
    if dist is None:
        return float(value)
    import torch
    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def algorithmic_bytes(n_sites, n_bonds, n_pairs, precision):
    """Bytes one reference step (i_step) must move, split by kernel.

    Sites are FP64: r read and written, the previous position and the
    projected noise read or written (96 B/site), all in the integrator.
    Bond geometry (centre, u, l) is written by the integrator and read by the
    pair kernel: 32 B mixed, 56 B FP64.  The per-bond force/torque
    accumulators are written by the pair kernel and read by the integrator:
    24 B mixed, 48 B FP64.  Each candidate pair costs 8 B of list read.
    Returns (integrator bytes, pair-kernel bytes) per launch."""
    geom, acc = (32, 24) if precision == "mixed" else (56, 48)
    integrate = 96 * n_sites + (geom + acc) * n_bonds
    pairs = (geom + acc) * n_bonds + 8 * n_pairs
    return integrate, pairs


def kernel_times(ctx, n):
    """Average CUDA-event duration (ms) of the pair kernel and of the
    integrator over n host-driven reference steps on the context's stream
    (L2 warm, as between the reference steps inside one timed launch)."""
    tp = ti = 0.0
    for _ in range(n):
        ctx.set_kernel_timing(True)
        ctx.interact()
        a, _ = ctx.kernel_timing()
        ctx.set_kernel_timing(True)
        ctx.update_positions()
        b, _ = ctx.kernel_timing()
        tp += a
        ti += b
    ctx.set_kernel_timing(False)
    return tp / n, ti / n


def profile_only(args):
    """--profile-steps N: host-driven reference steps of the bench workload
    (one pair launch and one integrator launch each) after 4 warm-up steps,
    nothing timed; the command the ncu captures run."""
    import simcore_b200 as sc
    from simcore_b200 import workloads
    system, fils, sites = workloads.make(args.workload, 1.0, seed=0)
    ctx = sc.Context(system, fils, sites, precision=args.precision, device=0)
    ctx.step(4)
    ctx.step(args.profile_steps)
    ctx.synchronize()
    c = ctx.counters()
    ctx.close()
    print(json.dumps({"profile_steps": args.profile_steps, "precision": args.precision,
                      "bonds": c.n_bonds, "pairs": c.n_pairs}))


def run_ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    import simcore_b200 as sc
    from simcore_b200 import workloads

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    system, fils, sites = workloads.make(args.workload, 1.0, seed=replica_seed(rank))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed_graph(ctx, k, flush_l2=True):
        """k bench steps; returns per-step device ms (CUDA events)."""
        out = []
        for _ in range(k):
            if flush_l2:
                flush.zero_()
                torch.cuda.synchronize()
            ctx.step_graph(I_STEPS_PER_STEP)
            out.append(ctx.graph_time_ms())
        return out

    results = {}
    contexts = {}
    layouts = {}
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(1.5)  # nvidia-smi needs a moment before its first sample
    for prec in ("fp64", "mixed"):
        ctx = sc.Context(system, fils, sites, precision=prec, device=local_rank)
        contexts[prec] = ctx
        layouts[prec] = ctx.autotune()  # integrator layout for this shape
        timed_graph(ctx, args.warmup)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        c0 = ctx.counters()
        t_start = time.perf_counter()
        ms = timed_graph(ctx, args.steps)
        torch.cuda.synchronize()
        if sampler:
            sampler.mark(t_start, time.perf_counter())
        c1 = ctx.counters()
        total_ms = reduce_max(float(sum(ms)), dist)
        results[prec] = dict(total_ms=total_ms, n_bonds=c1.n_bonds, n_sites=c1.n_sites,
                             n_pairs=c1.n_pairs, rebuilds=c1.n_rebuilds - c0.n_rebuilds,
                             launches=c1.kernel_launches - c0.kernel_launches)

    if sampler:
        results["clocks"] = sampler.stop()

    # Mixed-precision force error on this workload: fresh contexts of both
    # precisions on the initial positions evaluate the pair forces once; the
    # mixed bond forces and torques are compared with the FP64 ones
    # (max |dF| / max |F|).
    errs = {}
    for p_ in ("fp64", "mixed"):
        cc = sc.Context(system, fils, sites, precision=p_, device=local_rank)
        cc.interact()
        errs[p_] = cc.bond_forces()
        cc.close()
    force_err = float(np.abs(errs["mixed"][0] - errs["fp64"][0]).max() /
                      np.abs(errs["fp64"][0]).max())
    torque_err = float(np.abs(errs["mixed"][1] - errs["fp64"][1]).max() /
                       np.abs(errs["fp64"][1]).max())

    # Roofline: per-launch CUDA-event durations of the two kernels of a
    # reference step, host-driven, on the context's stream.
    kt = {p: kernel_times(contexts[p], 2 * I_STEPS_PER_STEP) for p in ("mixed", "fp64")}
    ctx = contexts["mixed"]

    # End to end through the C ABI with host buffers: every bench step
    # uploads the positions from pinned host memory, runs the 20 reference
    # steps and reads the positions back into pinned host memory.
    host_in = torch.empty((r_sites := ctx.n_sites, 3), dtype=torch.float64,
                          pin_memory=True).numpy()
    host_out = torch.empty((r_sites, 3), dtype=torch.float64, pin_memory=True).numpy()
    ctx.sites(out=host_in)
    for _ in range(args.warmup):
        ctx.set_sites(host_in)
        ctx.step_graph(I_STEPS_PER_STEP)
        ctx.sites(out=host_out)
        host_in, host_out = host_out, host_in
    e2e_times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.set_sites(host_in)
        ctx.step_graph(I_STEPS_PER_STEP)
        ctx.sites(out=host_out)
        e2e_times.append(time.perf_counter() - t0)
        host_in, host_out = host_out, host_in
    e2e_total = reduce_max(float(sum(e2e_times)), dist)

    for c in contexts.values():
        c.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    r = results["mixed"]
    r64 = results["fp64"]
    n_b = r["n_bonds"]
    seg_steps = n_b * I_STEPS_PER_STEP * args.steps * world
    value = seg_steps / (r["total_ms"] * 1e-3)
    value64 = seg_steps / (r64["total_ms"] * 1e-3)
    peak, peak_kind = load_measured_peaks()

    def roof(prec):
        rr = results[prec]
        b_int, b_pair = algorithmic_bytes(rr["n_sites"], rr["n_bonds"], rr["n_pairs"], prec)
        t_pair, t_int = kt[prec]
        return b_int, b_pair, t_pair, t_int

    b_int, b_pair, t_pair, t_int = roof("mixed")
    achieved = b_int / (t_int * 1e-3) / 1e9
    step_achieved = (b_int + b_pair) / ((t_int + t_pair) * 1e-3) / 1e9
    b_int64, b_pair64, t_pair64, t_int64 = roof("fp64")
    step64 = (b_int64 + b_pair64) / ((t_int64 + t_pair64) * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair forces + f64 integrator",
        "data": "synthetic (seeded random insertion with overlap rejection)",
        "config": {"workload": WORKLOAD_DESC, "precision": "mixed",
                   "i_steps_per_step": I_STEPS_PER_STEP,
                   "timed_unit": "one CUDA-graph launch of 20 reference steps (WHILE loop of 10 "
                                 "midpoint BD steps with device-decided pair-list rebuilds)",
                   "l2": "flushed by a 256 MiB write before every timed step",
                   "parallelism": "replicas" if world > 1 else "single system",
                   "pairs": r["n_pairs"], "rebuilds_in_timed_region": r["rebuilds"],
                   "integrator_layout": {p: {"warp_max_sites": w, "block_sites": b}
                                         for p, (w, b) in layouts.items()}},
        "fp64": {"value": value64, "ms_per_step": r64["total_ms"] / args.steps,
                 "rebuilds_in_timed_region": r64["rebuilds"]},
        "mixed_over_fp64": value / value64,
        "mixed_error": {"max_rel_bond_force": force_err, "max_rel_bond_torque": torque_err,
                        "vs": "FP64 GPU path (bit-identical to the reference) on the same "
                              "positions, one pair evaluation", "bound": 1e-5},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TRAFFIC_K_INTEGRATE_MIXED,
                     "kernel": "k_integrate<3,mixed,fast> (dominant: one launch per reference "
                               "step, all 20,000 filaments)",
                     "algorithmic_bytes_per_launch": b_int, "avg_launch_ms": t_int,
                     "peak_kind": peak_kind + " hbm_gbs",
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one "
                                       "launch of bench.py --profile-steps 8 (cold cache)",
                     "pair_kernel": {"kernel": "k_pair_eval (mixed)", "avg_launch_ms": t_pair,
                                     "algorithmic_bytes_per_launch": b_pair,
                                     "achieved": b_pair / (t_pair * 1e-3) / 1e9},
                     "reference_step": {"kernels": "k_pair_eval + k_integrate",
                                        "algorithmic_bytes": b_int + b_pair,
                                        "ms": t_int + t_pair, "achieved": step_achieved,
                                        "frac": step_achieved / peak},
                     "reference_step_fp64": {"algorithmic_bytes": b_int64 + b_pair64,
                                             "ms": t_int64 + t_pair64, "achieved": step64,
                                             "frac": step64 / peak}},
        "e2e": {"value": seg_steps / e2e_total, "unit": UNIT,
                "h2d_bytes_per_step": 24 * r["n_sites"], "d2h_bytes_per_step": 24 * r["n_sites"],
                "path": "sc_set_sites (pinned host -> device) + sc_step_graph(20) + "
                        "sc_get_sites (device -> pinned host), wall clock, max over ranks"},
        "gpu_launches": int(r["launches"]),
        "clocks": results.get("clocks"),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(system, fils, sites, n_b)
    return line


def cpu_baseline(system, fils, sites, n_bonds, target_s=10.0):
    """The reference's own code (oracle/_ref) on the same workload, OpenMP
    over all host cores; falls back to the single-threaded C oracle when the
    reference build is not present.  A bounded sample of steps."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import Oracle, Reference
    cores = host_cores()
    if Reference.available():
        sim = Reference(system, fils, sites, n_threads=cores)
        kind = "reference"
    else:
        sim = Oracle(system, fils, sites)
        kind, cores = "port", 1
    t0 = time.perf_counter()
    sim.step(2)
    dt = max(time.perf_counter() - t0, 1e-6)
    n = int(max(2, min(400, target_s / (dt / 2))))
    n += n % 2
    t0 = time.perf_counter()
    sim.step(n)
    el = time.perf_counter() - t0
    sim.close()
    return {"value": n_bonds * n / el, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": "%d reference steps of the same workload (after 2 warm-up steps)" % n}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import Reference
    from simcore_b200 import workloads
    if not Reference.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libscref.so (the reference's "
                "own sources) was not built on this machine"}
    system, fils, sites = workloads.make(args.workload, 1.0, seed=0)
    cores = host_cores()
    sim = Reference(system, fils, sites, n_threads=cores)
    n_b = sim.n_bonds
    # Size each bench step to a bounded sample: at most 20 reference steps,
    # fewer if one step is slow, so that warm-up + timed steps stay short.
    t0 = time.perf_counter()
    sim.step(2)
    per = max((time.perf_counter() - t0) / 2, 1e-6)
    budget_s = 150.0 / max(args.steps + args.warmup, 1)
    per_step = int(max(2, min(I_STEPS_PER_STEP, budget_s / per)))
    per_step -= per_step % 2
    for _ in range(args.warmup):
        sim.step(per_step)
    times = []
    for _ in range(args.steps):
        times.append(sim.step(per_step))
    sim.close()
    total = float(sum(times))
    value = n_b * per_step * args.steps / total
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random insertion with overlap rejection)",
        "config": {"workload": WORKLOAD_DESC, "i_steps_per_step": per_step,
                   "implementation": "reference C++ (object, site, bond, mesh, filament, cell, "
                                     "cell_list, minimum_distance, linear_algebra) -O3 OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "%d reference steps per bench step" % per_step},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    if args.profile_steps:
        profile_only(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
