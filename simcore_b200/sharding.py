"""Independent systems shared out over ranks (one process per GPU).

A batch of independent periodic systems (workload D: 256 replicas) needs no
communication while it runs: each rank loads a disjoint share of the systems
into one context of its own and steps it; per-system results are gathered
once at the end.  The reference runs such parameter sets one after another
in one process (SimulationManager::RunSimulations,
src/simulation_manager.cpp:537-553); here they run side by side, a share per
GPU and every system of a share in one launch per stage.

Shares balance the bonds per rank (longest processing time first: systems in
decreasing bond count, each to the rank with the fewest bonds so far, ties to
the lower rank), so the slowest rank -- whose time is the job's -- carries as
little as possible.  A system's results do not depend on which rank runs it:
its noise key, box and pair list are its own.
"""
import numpy as np


def partition(weights, world):
    """Indices of the systems each rank runs: a list of `world` ascending
    index lists covering range(len(weights)) once, balanced by weight."""
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0] * world
    shares = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(i)
        load[r] += weights[i]
    return [sorted(s) for s in shares]


def system_blocks(filaments, replicas, n_bonds):
    """Per system: (first filament, filament count, first site, site count,
    bond count), with n_bonds(params) the bond-count rule."""
    out, f0, s0 = [], 0, 0
    for rep in replicas:
        nf = rep["n_filaments"]
        nb = sum(n_bonds(f) for f in filaments[f0:f0 + nf])
        ns = nb + nf
        out.append((f0, nf, s0, ns, nb))
        f0 += nf
        s0 += ns
    return out


def share(system, filaments, sites, replicas, rank, world, n_bonds):
    """The sub-batch rank `rank` of `world` runs: (system, filaments, sites,
    replicas, indices), indices being the global numbers of its systems in
    the order it holds them.  An empty share has no filaments."""
    blocks = system_blocks(filaments, replicas, n_bonds)
    idx = partition([b[4] for b in blocks], world)[rank]
    fils, parts, reps = [], [], []
    for i in idx:
        f0, nf, s0, ns, _ = blocks[i]
        fils += filaments[f0:f0 + nf]
        parts.append(sites[s0:s0 + ns])
        reps.append(dict(replicas[i]))
    sub_sites = np.concatenate(parts) if parts else np.zeros((0, 3))
    sub_system = dict(system)
    if reps:
        sub_system.update(system_radius=reps[0]["system_radius"], seed=reps[0]["seed"])
    return sub_system, fils, sub_sites, reps, idx


def gather_by_system(values, indices, n_systems, dist=None):
    """Per-system values of every rank in global system order, on every
    rank: `values[k]` belongs to global system `indices[k]`.  dist is
    torch.distributed (one all_gather_object over the ranks) or None for a
    single process."""
    pairs = list(zip(indices, values))
    if dist is not None:
        everyone = [None] * dist.get_world_size()
        dist.all_gather_object(everyone, pairs)
        pairs = [p for part in everyone for p in part]
    out = [None] * n_systems
    for i, v in pairs:
        if out[i] is not None:
            raise ValueError("system %d reported by two ranks" % i)
        out[i] = v
    if any(v is None for v in out):
        raise ValueError("a system was not reported by any rank")
    return out
