"""Independent systems shared out over ranks (simcore_b200.sharding), on CPU.

The shares cover every system once and balance the bonds; two gloo ranks
each run their share of a small replica batch on the CPU oracle and gather
the per-system results, which must equal a one-process run system by
system (a system's results do not depend on the rank that runs it).
"""
import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_system_once_and_balances():
    from simcore_b200.sharding import partition
    rng = np.random.default_rng(1)
    w = list(rng.integers(200, 2000, 256) * 16)
    for world in (1, 2, 3, 8):
        shares = partition(w, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(256))
        loads = [sum(w[i] for i in s) for s in shares]
        # longest-processing-time-first: within one system of the mean
        assert max(loads) - sum(loads) / world <= max(w)
    assert partition([5, 5, 5], 5)[3:] == [[], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


N_STEPS = 40


def _run_systems(triples):
    """Final positions of each (system, filaments, sites) after N_STEPS on
    the CPU oracle."""
    from checkers import Oracle
    out = []
    for system, fils, sites in triples:
        o = Oracle(system, fils, sites)
        o.step(N_STEPS)
        out.append(o.sites())
        o.close()
    return out


def _batch():
    from checkers import oracle_insert, workloads_module
    return workloads_module().make_replicas("D", n_replicas=5, fil_scale=0.03, seed=9,
                                            insert=oracle_insert)


def _rank_main(rank, world, port, out_path):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import datetime

    import torch.distributed as dist

    from checkers import oracle_n_bonds, workloads_module
    from simcore_b200.sharding import gather_by_system, share
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        system, fils, sites, reps = _batch()
        sub_sys, sub_fils, sub_sites, sub_reps, idx = share(system, fils, sites, reps, rank,
                                                            world, oracle_n_bonds)
        triples = workloads_module().split_replicas(sub_sys, sub_fils, sub_sites, sub_reps,
                                                    n_bonds=oracle_n_bonds) if sub_reps else []
        mine = _run_systems(triples)
        everything = gather_by_system(mine, idx, len(reps), dist)
        if rank == 0:
            np.savez(out_path, *everything)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process(tmp_path):
    import torch.multiprocessing as mp

    from checkers import oracle_n_bonds, workloads_module
    out_path = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out_path), nprocs=2, join=True,
                       start_method="spawn")
    system, fils, sites, reps = _batch()
    single = _run_systems(workloads_module().split_replicas(system, fils, sites, reps,
                                                            n_bonds=oracle_n_bonds))
    got = np.load(out_path)
    assert len(got.files) == len(single) == 5
    for k, want in enumerate(single):
        assert np.array_equal(got["arr_%d" % k], want), k
