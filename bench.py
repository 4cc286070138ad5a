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
independent replica (weak scaling, no data-path collective); with --workload
D the 256 independent systems are shared out over the ranks instead (strong
scaling; per-system counts gathered once at the end).  The time is the max
over ranks.  --impl reference times the reference's own CPU code
(oracle/_ref, OpenMP over all host cores) on the same configuration, made by
the oracle's insertion, without loading the CUDA library.
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
# Points of the timed mixed trajectory at which the mixed-precision error is
# measured (after every quarter of the timed steps).
N_SNAPSHOTS = 4
# DRAM bytes (read + write) of one k_integrate launch, mixed precision, from
# ncu (cold cache), per workload captured, with the block layout the timed
# runs use: for B (192-site blocks) the mean of a midstep launch (22.11 MB)
# and a full-step launch (39.73 MB), which alternate.  Workloads without a
# capture report null.
TRAFFIC_K_INTEGRATE_MIXED = {"B": 30.92e6}
TRAFFIC_LAYOUT = {"B": "0,192"}
WORKLOAD_DESCS = {
    "A": "A: 100 filaments x 20 bonds (2,000 segments, 2,100 sites), 3D periodic cube side 50, "
         "lp 500, WCA eps=sigma=1, dt 1e-4, noise on",
    "B": "B: 20,000 filaments x 10 bonds (200,000 segments, 220,000 sites), 3D periodic cube side "
         "200, lp 100, WCA eps=sigma=1, dt 1e-4, noise on",
    "C": "C: 50,000 filaments x log-uniform[5,200] bonds (2.64M segments), lp uniform[10,1000], "
         "3D periodic cube side 300, WCA eps=sigma=1, dt 5e-5, noise on",
    "D": "D: 256 independent 2D periodic systems of uniform[200,2000] filaments x 16 bonds "
         "(4.5M segments), area fraction 0.1, lp 200, WCA eps=sigma=1, dt 1e-4, noise on, "
         "one context",
    "E": "E: 10,000 filaments x 50 bonds (500,000 segments), 3D periodic cube side 150, lp 1000, "
         "100,000 static tethers k=10 rest 1, WCA eps=sigma=1, dt 1e-4, noise on",
}
WORKLOAD_DESC = WORKLOAD_DESCS["B"]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 200 launches of 20 reference steps: about 0.3 s per precision on B,
    # long enough for a few dozen clock samples of the timed region.
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="B", choices=sorted(WORKLOAD_DESCS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many host-driven steps and exit (for ncu)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of --profile-steps")
    ap.add_argument("--layout-sweep", action="store_true",
                    help="time every integrator layout of the workload (one JSON line each) "
                         "and exit")
    ap.add_argument("--profile-fused", action="store_true",
                    help="--profile-steps with the pair evaluation fused into the integrator")
    ap.add_argument("--profile-layout", default=None,
                    help="integrator layout W,C for --profile-steps (warp-kernel sites, block "
                         "sites), e.g. the one the timed run's autotuner chose")
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


def reduce_sum(value, dist):
    """Sum over ranks; dist may be None."""
    if dist is None:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
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


def fused_bytes(n_sites, n_bonds, n_pairs):
    """Bytes of one launch of the mixed integrator with the pair evaluation
    fused in: the sites' 96 B, the bond geometry this step reads (32 B) and
    the one it writes for the next (32 B), and 8 B of list per candidate pair.
    The pair stage's per-bond accumulators are neither written nor read."""
    return 96 * n_sites + 64 * n_bonds + 8 * n_pairs


def step_kernel_time(ctx, n):
    """Average CUDA-event duration (ms) of the kernels sc_step launches for a
    reference step, over n host-driven steps (L2 warm): with
    sc_set_fused_pairs on (fast mixed step), the integrator with the pairs
    fused in, alone."""
    t = 0.0
    for _ in range(n):
        ctx.set_kernel_timing(True)
        ctx.step(1)
        a, _ = ctx.kernel_timing()
        t += a
    ctx.set_kernel_timing(False)
    return t / n


def kernel_times(ctx, n):
    """Average CUDA-event duration (ms) of the pair kernel and of the
    integrator over n host-driven reference steps of the split interface
    (sc_interact, then sc_update_positions) on the context's stream (L2
    warm, as between the reference steps inside one timed launch)."""
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


def load_workload(name, seed):
    """(system, filaments, sites, replicas, crosslinks) of a workload, made by
    the library's insertion."""
    from simcore_b200 import workloads
    if name == "D":
        system, fils, sites, reps = workloads.make_replicas("D", seed=seed)
        return system, fils, sites, reps, None
    system, fils, sites = workloads.make(name, 1.0, seed=seed)
    xl = workloads.crosslinks(name, sites, fils, 2 * system["system_radius"], seed=seed)
    return system, fils, sites, None, xl


def workload_config(name):
    """The `config` of both arms' JSON lines: the workload and the units of
    the metric, nothing that depends on the arm."""
    return {"workload": WORKLOAD_DESCS[name],
            "segment": "one bond of a filament",
            "step": "one reference i_step: a pair-force evaluation and an integrator half "
                    "step, delta/2 of simulated time"}


def new_context(sc, wl, prec, device):
    system, fils, sites, reps, xl = wl
    ctx = sc.Context(system, fils, sites, precision=prec, device=device, replicas=reps)
    if xl is not None:
        a, b, k, rest = xl
        ctx.add_crosslinks(a, b, k_spring=k, rest_length=rest)
    return ctx


def cpu_runs(wl, cores):
    """CPU simulations of a workload for the baseline: the reference's own
    code (oracle/_ref, OpenMP on `cores` threads, its own Crosslink and
    Anchor code for tethered networks), or the C oracle on one thread where
    oracle/_ref was not built.  Independent systems run one after another
    (the reference keeps static state: one simulation per process at a time),
    a leading subset of them.  Returns (kind, cores, [(make, bonds)], note),
    make() creating one simulation.  Uses the CPU checkers only (bond counts
    by the oracle's rule): the CUDA library is not loaded here."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import Oracle, Reference, oracle_n_bonds, workloads_module
    system, fils, sites, reps, xl = wl
    bonds = lambda fs: sum(oracle_n_bonds(f) for f in fs)
    use_ref = Reference.available()
    kind, cores = ("reference", cores) if use_ref else ("port", 1)
    make = (lambda *a: Reference(*a, n_threads=cores)) if use_ref else Oracle
    if xl is not None:
        def make_tethered():
            sim = make(system, fils, sites)
            sim.add_crosslinks(xl[0], xl[1], k_spring=xl[2], rest_length=xl[3])
            return sim
        return kind, cores, [(make_tethered, bonds(fils))], \
            "with the crosslinks attached by the reference's own code" if use_ref else \
            "C oracle with the restated tethers (1 thread)"
    if reps is None:
        if bonds(fils) <= 1000000:
            return kind, cores, [(lambda: make(system, fils, sites), bonds(fils))], ""
        # A bounded sample: the first filaments, up to 100,000 bonds, in the
        # full box.  (The reference's set-up of the full system -- its cell
        # list and per-filament storage -- takes longer than the whole
        # default bench run.)
        n_keep, nb_keep = 0, 0
        while n_keep < len(fils) and nb_keep < 100000:
            nb_keep += oracle_n_bonds(fils[n_keep])
            n_keep += 1
        ns_keep = nb_keep + n_keep
        sub = (system, fils[:n_keep], sites[:ns_keep])
        return kind, cores, [(lambda: make(*sub), nb_keep)], \
            "the first %d of %d filaments in the full box" % (n_keep, len(fils))
    runs, total = [], 0
    for part in workloads_module().split_replicas(system, fils, sites, reps,
                                                  n_bonds=oracle_n_bonds):
        runs.append(((lambda p=part: make(*p)), bonds(part[1])))
        total += runs[-1][1]
        if total >= 100000:
            break
    return kind, cores, runs, "the first %d of %d systems, one after another" % (len(runs), len(reps))


def profile_only(args):
    """--profile-steps N: host-driven reference steps of the bench workload
    (a pair launch and an integrator launch each; with --profile-fused, mixed,
    one integrator launch with the pairs fused in) after 4 warm-up steps,
    nothing timed; the command the ncu captures run."""
    import simcore_b200 as sc
    from simcore_b200 import workloads
    ctx = new_context(sc, load_workload(args.workload, 0), args.precision, 0)
    layout = None
    if args.profile_layout:
        layout = [int(v) for v in args.profile_layout.split(",")]
        ctx.set_integrator_layout(*layout)
    if args.profile_fused:
        ctx.set_exact_near_parallel(False)
        ctx.set_fused_pairs(True)
    ctx.step(4)
    ctx.step(args.profile_steps)
    ctx.synchronize()
    c = ctx.counters()
    ctx.close()
    print(json.dumps({"profile_steps": args.profile_steps, "precision": args.precision,
                      "layout": layout, "bonds": c.n_bonds, "pairs": c.n_pairs}))


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

    scaling = "weak"
    shard = None
    if args.workload == "D" and world > 1:
        # The 256 independent systems are shared out over the ranks, balanced
        # by bonds (simcore_b200.sharding); each rank makes and runs only its
        # share, and the total work is fixed.
        from simcore_b200 import sharding
        counts = workloads.replica_counts("D")
        n_seg = workloads.REPLICAS["D"]["n_seg"]
        shard = sharding.partition([int(c) * n_seg for c in counts], world)[rank]
        system, fils, sites, reps = workloads.make_replicas("D", only=shard)
        wl = (system, fils, sites, reps, None)
        scaling = "strong"
    else:
        wl = load_workload(args.workload, replica_seed(rank))
    system, fils, sites = wl[:3]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed_graph(ctx, k, flush_l2=True, snapshots=None):
        """k bench steps; returns per-step device ms (CUDA events).  With a
        list `snapshots`, the positions after every quarter of the steps are
        appended to it (read between launches, outside the timed launches)."""
        out = []
        marks = {max(1, (k * q) // N_SNAPSHOTS) for q in range(1, N_SNAPSHOTS + 1)}
        for i in range(k):
            if flush_l2:
                flush.zero_()
                torch.cuda.synchronize()
            ctx.step_graph(I_STEPS_PER_STEP)
            out.append(ctx.graph_time_ms())
            if snapshots is not None and i + 1 in marks:
                snapshots.append((ctx.counters().i_step, ctx.sites()))
        return out

    results = {}
    contexts = {}
    layouts = {}
    snaps = []  # (i_step, positions) along the timed mixed-precision trajectory
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(1.5)  # nvidia-smi needs a moment before its first sample
    for prec in ("fp64", "mixed"):
        ctx = new_context(sc, wl, prec, local_rank)
        contexts[prec] = ctx
        layouts[prec] = ctx.autotune()  # integrator layout for this shape
        timed_graph(ctx, args.warmup)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        c0 = ctx.counters()
        t_start = time.perf_counter()
        ms = timed_graph(ctx, args.steps, snapshots=snaps if prec == "mixed" else None)
        torch.cuda.synchronize()
        if sampler:
            sampler.mark(t_start, time.perf_counter())
        c1 = ctx.counters()
        total_ms = reduce_max(float(sum(ms)), dist)
        results[prec] = dict(total_ms=total_ms, n_bonds=c1.n_bonds, n_sites=c1.n_sites,
                             n_fil=c1.n_filaments, n_dim=wl[0]["n_dim"], n_pairs=c1.n_pairs, rebuilds=c1.n_rebuilds - c0.n_rebuilds,
                             launches=c1.kernel_launches - c0.kernel_launches)

    if sampler:
        results["clocks"] = sampler.stop()

    # Mixed precision against FP64, output by output (simcore_b200.accuracy):
    # fresh contexts of both precisions on the same positions -- the inserted
    # state and the snapshots of the timed mixed trajectory -- evaluate the
    # pair forces and one integrator step with shared noise.
    from simcore_b200.accuracy import max_errors, mixed_errors
    sysd, fl, _, reps_, xl_ = wl
    err_inserted = mixed_errors(sysd, fl, wl[2], reps_, xl_, device=local_rank)
    err_traj = [dict(mixed_errors(sysd, fl, xyz, reps_, xl_, device=local_rank), i_step=ist)
                for ist, xyz in snaps]
    err_max = max_errors([err_inserted] + err_traj)

    # Roofline: per-launch CUDA-event durations of the two kernels of a
    # reference step, host-driven, on the context's stream; beside them the
    # integrator with the pairs fused in (sc_set_fused_pairs, off in the
    # timed runs).
    kt = {p: kernel_times(contexts[p], 2 * I_STEPS_PER_STEP) for p in ("mixed", "fp64")}
    ctx = contexts["mixed"]
    ctx.set_exact_near_parallel(False)  # the fusion evaluates every pair in FP32
    ctx.set_fused_pairs(True)
    t_fused = step_kernel_time(ctx, 2 * I_STEPS_PER_STEP)
    ctx.set_fused_pairs(False)
    ctx.set_exact_near_parallel(True)

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

    per_system = None
    if shard is not None:
        # Per-system rebuild and pair counts of the mixed run, gathered from
        # every rank in global system order.
        from simcore_b200 import sharding
        nr, npr = contexts["mixed"].replica_counters()
        rows = [(int(a), int(b)) for a, b in zip(nr, npr)]
        gathered = sharding.gather_by_system(rows, shard, len(workloads.replica_counts("D")),
                                             dist)
        per_system = {"systems": len(gathered),
                      "rebuilds_total": sum(g[0] for g in gathered),
                      "pairs_total": sum(g[1] for g in gathered),
                      "systems_per_rank_this_rank": len(shard)}
    for c in contexts.values():
        c.close()
    r = results["mixed"]
    r64 = results["fp64"]
    # Segment-steps of every rank (shares of independent systems differ in
    # size); the time is the slowest rank's.
    seg_steps = reduce_sum(r["n_bonds"] * I_STEPS_PER_STEP * args.steps, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    n_b = r["n_bonds"]
    value = seg_steps / (r["total_ms"] * 1e-3)
    value64 = seg_steps / (r64["total_ms"] * 1e-3)
    peak, peak_kind = load_measured_peaks()

    def roof(prec):
        rr = results[prec]
        b_int, b_pair = algorithmic_bytes(rr["n_sites"], rr["n_bonds"], rr["n_pairs"], prec)
        t_pair, t_int = kt[prec]
        return b_int, b_pair, t_pair, t_int

    b_int, b_pair, t_pair, t_int = roof("mixed")
    b_fused = fused_bytes(r["n_sites"], r["n_bonds"], r["n_pairs"])
    achieved = b_int / (t_int * 1e-3) / 1e9
    step_achieved = (b_int + b_pair) / ((t_int + t_pair) * 1e-3) / 1e9
    b_int64, b_pair64, t_pair64, t_int64 = roof("fp64")
    step64 = (b_int64 + b_pair64) / ((t_int64 + t_pair64) * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": scaling, "vs_baseline": None, "dtype": "f32 pair forces + f64 integrator",
        "data": "synthetic (seeded random insertion with overlap rejection)",
        "config": workload_config(args.workload),
        "run": {"precision": "mixed", "i_steps_per_step": I_STEPS_PER_STEP,
                "timed_unit": "one CUDA-graph launch of 20 reference steps (WHILE loop of 10 "
                              "midpoint BD steps with device-decided pair-list rebuilds)",
                "l2": "flushed by a 256 MiB write before every timed step",
                "parallelism": ("independent systems shared out over %d ranks" % world
                                if shard is not None else
                                "replicas" if world > 1 else "single system"),
                "per_system": per_system,
                "pairs": r["n_pairs"], "rebuilds_in_timed_region": r["rebuilds"],
                "integrator_layout": {p: {"warp_max_sites": w, "block_sites": b}
                                      for p, (w, b) in layouts.items()}},
        "fp64": {"value": value64, "ms_per_step": r64["total_ms"] / args.steps,
                 "rebuilds_in_timed_region": r64["rebuilds"]},
        "mixed_over_fp64": value / value64,
        "mixed_error": {
            "bound": 1e-5, "max": err_max, "inserted_state": err_inserted,
            "trajectory": err_traj,
            "vs": "FP64 GPU path (bit-identical to the reference) on the same positions: "
                  "fresh contexts of both precisions evaluate the pair forces and one "
                  "integrator step with shared noise; max |mixed - fp64| / max |fp64| per "
                  "output (displacement = positions after the step - before)",
            "states": "the inserted state and the timed mixed trajectory after every "
                      "quarter of the timed steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": TRAFFIC_K_INTEGRATE_MIXED.get(args.workload),
                     "kernel": "k_integrate<%d,mixed,fast> (dominant: one launch per reference "
                               "step, all %d filaments)" % (r["n_dim"], r["n_fil"]),
                     "algorithmic_bytes_per_launch": b_int, "avg_launch_ms": t_int,
                     "peak_kind": peak_kind + " hbm_gbs",
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, mean "
                                       "of a midstep and a full-step launch of bench.py "
                                       "--profile-steps 8 --profile-layout %s (cold cache)"
                                       % TRAFFIC_LAYOUT.get(args.workload, "-"),
                     "pair_kernel": {"kernel": "k_pair_eval (mixed)", "avg_launch_ms": t_pair,
                                     "algorithmic_bytes_per_launch": b_pair,
                                     "achieved": b_pair / (t_pair * 1e-3) / 1e9},
                     "reference_step": {"kernels": "k_pair_eval + k_integrate",
                                        "algorithmic_bytes": b_int + b_pair,
                                        "ms": t_int + t_pair, "achieved": step_achieved,
                                        "frac": step_achieved / peak},
                     "fused_pairs_option": {
                         "kernel": "k_integrate<%d,mixed,fast,fused pairs> (sc_set_fused_pairs, "
                                   "all pairs in FP32; off in the timed runs)" % r["n_dim"],
                         "avg_launch_ms": t_fused, "algorithmic_bytes_per_launch": b_fused,
                         "achieved": b_fused / (t_fused * 1e-3) / 1e9},
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
        line["cpu_baseline"] = cpu_baseline(wl)
    return line


def cpu_baseline(wl, target_s=10.0):
    """The reference's CPU code on the same workload (cpu_runs), a bounded
    sample of steps sized to about target_s seconds in all."""
    kind, cores, runs, note = cpu_runs(wl, host_cores())
    seg, el, n_used = 0, 0.0, 0
    for make, nb in runs:
        sim = make()
        t0 = time.perf_counter()
        sim.step(2)
        dt = max(time.perf_counter() - t0, 1e-6)
        n = int(max(2, min(400, target_s / len(runs) / (dt / 2))))
        n += n % 2
        t0 = time.perf_counter()
        sim.step(n)
        el += time.perf_counter() - t0
        seg += nb * n
        n_used = max(n_used, n)
        sim.close()
    sample = "up to %d reference steps of the same workload (after 2 warm-up steps)" % n_used
    if note:
        sample += "; " + note
    return {"value": seg / el, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import Reference
    if not Reference.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libscref.so (the reference's "
                "own sources) was not built on this machine"}
    from checkers import oracle_workload
    # The GPU arm's configuration, made by the oracle's insertion (bit for
    # bit the library's): nothing of the CUDA library is loaded in this arm.
    kind, cores, runs, note = cpu_runs(oracle_workload(args.workload, 0), host_cores())
    # Size each bench step to a bounded sample: at most 20 reference steps,
    # fewer if one step is slow, so that warm-up + timed steps stay short.
    # (The first system's simulation, built once -- the reference's set-up
    # of a large box takes longer than its steps -- also runs its chunks.)
    first = runs[0][0]()
    t0 = time.perf_counter()
    first.step(2)
    per = max((time.perf_counter() - t0) / 2, 1e-6) * sum(nb for _, nb in runs) / runs[0][1]
    budget_s = 150.0 / max(args.steps + args.warmup, 1)
    per_step = int(max(2, min(I_STEPS_PER_STEP, budget_s / per)))
    per_step -= per_step % 2
    # Bench step k is the k-th chunk of per_step steps of every system.
    times = [0.0] * args.steps
    seg = 0
    for idx, (make, nb) in enumerate(runs):
        sim = first if idx == 0 else make()
        for _ in range(args.warmup):
            sim.step(per_step)
        for k in range(args.steps):
            t0 = time.perf_counter()
            sim.step(per_step)
            times[k] += time.perf_counter() - t0
            seg += nb * per_step
        sim.close()
    total = float(sum(times))
    value = seg / total
    sample = "%d reference steps per bench step" % per_step + ("; " + note if note else "")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random insertion with overlap rejection)",
        "config": workload_config(args.workload),
        "run": {"i_steps_per_step": per_step,
                "implementation": ("reference C++ (object, site, bond, mesh, filament, cell, "
                                   "cell_list, minimum_distance, linear_algebra) -O3 OpenMP"
                                   if kind == "reference" else
                                   "C restatement of the reference (tethers included)"),
                "inputs": "the GPU arm's initial configuration, made by the oracle's insertion"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def layout_sweep(args):
    """--layout-sweep: for both precisions and every integrator layout that
    holds the workload (warp kernel on or off, blocks of 64-256 sites), the
    CUDA-event time of the pair and integrator kernels of a host-driven
    reference step (L2 warm) and of a captured 20-step launch (L2 flushed
    first); one JSON line per layout.  Layouts are what sc_autotune chooses
    among; this prints all of their times."""
    import torch
    import simcore_b200 as sc
    wl = load_workload(args.workload, 0)
    n_sites = [sc.filament_n_bonds(f) + 1 for f in wl[1]]
    longest, shortest = max(n_sites), min(n_sites)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for prec in ("mixed", "fp64"):
        ctx = new_context(sc, wl, prec, 0)
        for w in (32, 0):
            if w == 32 and shortest > 32:
                continue
            rest = longest if (w == 0 or longest > 32) else 0
            for bsz in ((0,) if rest == 0 else (64, 96, 128, 160, 192, 256)):
                if rest and bsz < rest:
                    continue
                ctx.set_integrator_layout(w, bsz)
                t_pair, t_int = kernel_times(ctx, 2 * I_STEPS_PER_STEP)
                ms = []
                for i in range(3 + args.steps):
                    flush.zero_()
                    torch.cuda.synchronize()
                    ctx.step_graph(I_STEPS_PER_STEP)
                    if i >= 3:
                        ms.append(ctx.graph_time_ms())
                print(json.dumps({"precision": prec, "warp_max_sites": w, "block_sites": bsz,
                                  "pair_ms": t_pair, "integrate_ms": t_int,
                                  "graph_ms_per_20_steps": statistics.mean(ms)}), flush=True)
        ctx.close()


def main():
    args = parse_args()
    if args.profile_steps:
        profile_only(args)
        return
    if args.layout_sweep:
        layout_sweep(args)
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
