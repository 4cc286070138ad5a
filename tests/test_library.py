"""Host-side checks of the product library (no GPU needed).

The C ABI library loads and exports every symbol include/simcore_gpu.h
declares; without a device sc_create reports SC_ERR_NO_DEVICE; the host
insertion routine produces the reference's bond count and non-overlapping
filaments; the bench's replica reduction works across gloo ranks.
"""
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT


def test_header_symbols_are_exported():
    import simcore_b200 as sc
    header = open(os.path.join(ROOT, "include", "simcore_gpu.h")).read()
    declared = set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", header))
    assert declared == set(sc.EXPORTED)
    for name in declared:
        assert hasattr(sc.lib, name), name


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_create_without_device_reports_no_device():
    import simcore_b200 as sc
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("A", 0.1)
    with pytest.raises(sc.ScError) as e:
        sc.Context(system, fils, sites)
    assert e.value.code == 9


def test_filament_bond_count_rule():
    import simcore_b200 as sc
    for L in (5, 10, 20, 50, 200):
        p = dict(length=float(L), persistence_length=10.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)
        assert sc.filament_n_bonds(p) == L  # floor(L / 0.999)
    p = dict(length=3.0, persistence_length=10.0, diameter=1.0, min_bond_length=1.5,
             friction_ratio=2.0)
    assert sc.filament_n_bonds(p) == 2  # length clamped to 5, floor(5/2.25) = 2


def _min_segment_distance(sites, n_sites, L):
    from checkers import Oracle  # noqa: F401
    a = []
    off = 0
    for n in n_sites:
        for j in range(n - 1):
            a.append((sites[off + j], sites[off + j + 1], len(a), off))
        off += n
    best = np.inf
    for i in range(len(a)):
        for k in range(i + 1, len(a)):
            if a[i][3] == a[k][3]:
                continue  # same filament: not checked by insertion
            p1, p2 = a[i][0], a[i][1]
            q1, q2 = a[k][0], a[k][1]
            # sample-based distance check is enough to catch overlaps
            for s in np.linspace(0, 1, 6):
                pt = p1 + s * (p2 - p1)
                for u in np.linspace(0, 1, 6):
                    qt = q1 + u * (q2 - q1)
                    d = pt - qt
                    d -= L * np.round(d / L)
                    best = min(best, np.linalg.norm(d))
    return best


def test_insertion_geometry():
    import simcore_b200 as sc
    nb = np.full(12, 8, dtype=np.int32)
    sites = sc.insert_filaments(3, 8.0, 5, nb, nb.astype(float), np.full(12, 20.0))
    assert sites.shape == (12 * 9, 3)
    bl = np.linalg.norm(np.diff(sites.reshape(12, 9, 3), axis=1), axis=2)
    assert np.allclose(bl, 1.0, atol=1e-12)
    assert _min_segment_distance(sites, [9] * 12, 16.0) >= 1.0 - 1e-9


def _replica_rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    t = bench.reduce_max(float(10 + rank), dist)
    q.put((rank, t, bench.replica_seed(rank)))
    dist.destroy_process_group()


def test_replicas_reduce_max_over_gloo_ranks():
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [11.0, 11.0]
    assert got[0][2] != got[1][2]  # each replica its own seed


def test_workload_E_crosslinks():
    """Tethers of workload E: distinct site pairs within reach (minimum
    image), never the same or adjacent sites of one filament."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("E", scale=0.01, seed=1, n_seg=10)
    side = 2 * system["system_radius"]
    a, b, k, rest = workloads.crosslinks("E", sites, fils, side, scale=0.01, seed=1)
    assert 100 < len(a) <= 1000 and k == 10.0 and rest == 1.0
    d = sites[a] - sites[b]
    d -= side * np.round(d / side)
    assert np.all(np.sqrt((d ** 2).sum(1)) < 2.0)
    fil = np.repeat(np.arange(len(fils)), 11)
    assert not np.any((fil[a] == fil[b]) & (np.abs(a - b) <= 1))
    assert len(set(zip(a.tolist(), b.tolist()))) == len(a)
