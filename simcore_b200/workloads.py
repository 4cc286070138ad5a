"""Synthetic workloads of the filament step.

Every workload is a 3D (or 2D) periodic box of semiflexible filaments with
bond length 1 sigma (min_bond_length 0.666 makes floor(L / 0.999) = L bonds
for every integer length L, reference src/filament.cpp:142-147), diameter 1,
friction ratio 2, WCA eps = sigma = 1 with f_cutoff 2000, thermal noise on.
Initial configurations come from seeded random insertion with overlap
rejection (sc_insert_filaments); no dataset is involved.

  A  100 x 20 bonds, lp 500, side 50, dt 1e-4          (CPU parity case)
  B  20,000 x 10 bonds, lp 100, side 200, dt 1e-4       (dense suspension)
  C  50,000 x log-uniform[5,200] bonds, lp U[10,1000], side 300, dt 5e-5
     (its 100-200-bond filaments have an excluded volume several times the
     box: isotropic insertion cannot place them, so random_nematic)
  D  256 independent 2D systems (make_replicas): N_r ~ U{200..2000}
     filaments x 16 bonds, side sqrt(N_r (16 + pi/4) / 0.1), lp 200, dt 1e-4
  E  10,000 x 50 bonds, lp 1000, side 150, dt 1e-4      (network geometry;
     volume fraction 0.116 is above the isotropic-nematic point of 50:1 rods,
     so the filaments are inserted straight along -+z, random_nematic)
     plus 100,000 static tethers, k 10, rest length 1 (crosslinks())

scale < 1 shrinks the filament count and the box volume together (same
density) for parity tests at small sizes.

The module needs only numpy.  The library is imported when a workload is
made, for its insertion and bond-count rule, unless the caller passes its own
(`insert`, `n_bonds`): a CPU checker can then build the same configuration
without loading the CUDA library.
"""
import math

import numpy as np


def _library_insert(*args, **kw):
    from simcore_b200 import insert_filaments
    return insert_filaments(*args, **kw)


def _library_n_bonds(params):
    from simcore_b200 import filament_n_bonds
    return filament_n_bonds(params)

MIN_BOND_LENGTH = 0.666
DIAMETER = 1.0
FRICTION_RATIO = 2.0

WORKLOADS = {
    "A": dict(n_dim=3, side=50.0, n_fil=100, n_seg=20, lp=500.0, delta=1e-4, n_steps=1000),
    "B": dict(n_dim=3, side=200.0, n_fil=20000, n_seg=10, lp=100.0, delta=1e-4, n_steps=2000),
    "C": dict(n_dim=3, side=300.0, n_fil=50000, n_seg=("loguniform", 5, 200),
              lp=("uniform", 10.0, 1000.0), delta=5e-5, n_steps=1000,
              insertion="random_nematic"),
    "E": dict(n_dim=3, side=150.0, n_fil=10000, n_seg=50, lp=1000.0, delta=1e-4, n_steps=1000,
              insertion="random_nematic"),
}


CROSSLINKS = {"E": dict(n_links=100000, k_spring=10.0, rest_length=1.0, reach=2.0)}


def crosslinks(name, sites, filaments, side, scale=1.0, seed=0, n_bonds=None):
    """Static tethers of workload `name`: site pairs drawn uniformly from all
    pairs closer than `reach` (minimum image) that are not the same or
    adjacent sites of one filament.  Returns (site_a, site_b, k_spring,
    rest_length), or None for a workload without crosslinks."""
    if name not in CROSSLINKS:
        return None
    from scipy.spatial import cKDTree
    c = CROSSLINKS[name]
    n_dim = 3 if np.any(sites[:, 2] != 0) else 2
    pts = np.mod(sites[:, :n_dim], side)
    pts[pts >= side] = 0.0
    tree = cKDTree(pts, boxsize=side)
    pairs = tree.query_pairs(c["reach"], output_type="ndarray")
    n_bonds = n_bonds or _library_n_bonds
    n_sites = np.array([n_bonds(f) + 1 for f in filaments])
    fil = np.repeat(np.arange(len(filaments)), n_sites)
    same = (fil[pairs[:, 0]] == fil[pairs[:, 1]]) & (np.abs(pairs[:, 0] - pairs[:, 1]) <= 1)
    pairs = pairs[~same]
    d = sites[pairs[:, 0], :n_dim] - sites[pairs[:, 1], :n_dim]
    d -= side * np.round(d / side)
    pairs = pairs[np.einsum("ij,ij->i", d, d) < c["reach"] ** 2]  # strictly closer
    pairs = pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]
    n = min(len(pairs), max(1, int(round(c["n_links"] * scale))))
    rng = np.random.default_rng(seed + 777)
    pick = pairs[rng.choice(len(pairs), size=n, replace=False)]
    return (pick[:, 0].astype(np.int32), pick[:, 1].astype(np.int32), c["k_spring"],
            c["rest_length"])


REPLICAS = {"D": dict(n_dim=2, n_replicas=256, n_fil=(200, 2000), n_seg=16, lp=200.0,
                      area_fraction=0.1, delta=1e-4, n_steps=500)}


def replica_counts(name="D", n_replicas=None, fil_scale=1.0, seed=0):
    """Filament count of every system of make_replicas (same arguments)."""
    w = REPLICAS[name]
    nrep = w["n_replicas"] if n_replicas is None else int(n_replicas)
    rng = np.random.default_rng(seed + 4242)
    lo, hi = w["n_fil"]
    return np.maximum(2, np.round(rng.integers(lo, hi + 1, nrep) * fil_scale)).astype(int)


def make_replicas(name="D", n_replicas=None, fil_scale=1.0, seed=0, stoch=True,
                  interaction=True, insert=None, only=None):
    """Independent systems of workload `name`: returns (system, filaments,
    sites, replicas) for Context(..., replicas=replicas).  System r has
    N_r = round(U{lo..hi} * fil_scale) filaments (at least 2) in a periodic
    square of area N_r (n_seg + pi/4) / area_fraction (the reference's 2D
    filament area, src/filament.cpp:385-388), noise seed seed * 1000 + r.
    only: the indices of the systems to make (each is the same system it is
    in the whole batch), in that order; default all."""
    w = REPLICAS[name]
    counts = replica_counts(name, n_replicas, fil_scale, seed)
    fil_area = w["n_seg"] + math.pi / 4
    insert = insert or _library_insert
    filaments, blocks, replicas = [], [], []
    for r in (range(len(counts)) if only is None else only):
        n = int(counts[r])
        side = math.sqrt(n * fil_area / w["area_fraction"])
        n_seg = np.full(n, w["n_seg"], dtype=np.int32)
        lengths = n_seg.astype(np.float64)
        lp = np.full(n, w["lp"])
        rseed = seed * 1000 + r
        blocks.append(insert(w["n_dim"], 0.5 * side, rseed, n_seg, lengths, lp,
                             diameter=DIAMETER))
        filaments += [dict(length=float(lengths[i]), persistence_length=float(lp[i]),
                           diameter=DIAMETER, min_bond_length=MIN_BOND_LENGTH,
                           friction_ratio=FRICTION_RATIO) for i in range(n)]
        replicas.append(dict(system_radius=0.5 * side, seed=rseed, n_filaments=n))
    system = dict(n_dim=w["n_dim"], system_radius=replicas[0]["system_radius"],
                  delta=w["delta"], wca_eps=1.0, wca_sig=1.0, f_cutoff=2000.0,
                  stoch_flag=1 if stoch else 0, interaction_flag=1 if interaction else 0,
                  like_like_interactions=1, seed=replicas[0]["seed"])
    return system, filaments, np.concatenate(blocks), replicas


def split_replicas(system, filaments, sites, replicas, n_bonds=None):
    """Per-system (system, filaments, sites) triples of a replica batch, each
    as a stand-alone configuration."""
    n_bonds = n_bonds or _library_n_bonds
    out, f0, s0 = [], 0, 0
    for rep in replicas:
        fils = filaments[f0:f0 + rep["n_filaments"]]
        ns = sum(n_bonds(f) + 1 for f in fils)
        out.append((dict(system, system_radius=rep["system_radius"], seed=rep["seed"]), fils,
                    sites[s0:s0 + ns]))
        f0 += rep["n_filaments"]
        s0 += ns
    return out


def describe(name):
    w = WORKLOADS[name]
    return dict(w)


def make(name, scale=1.0, seed=0, precision_seed=None, stoch=True, interaction=True,
         n_seg=None, side=None, insert=None):
    """Returns (system, filaments, sites) for workload `name`.  For small test
    systems that full-length filaments would not fit: n_seg replaces the
    bonds per filament, side the box side (lower density)."""
    w = WORKLOADS[name]
    n_fil = max(2, int(round(w["n_fil"] * scale)))
    if side is None:
        side = w["side"] * (scale ** (1.0 / w["n_dim"]))
    rng = np.random.default_rng(seed + 12345)
    seg = w["n_seg"] if n_seg is None else int(n_seg)
    if isinstance(seg, tuple):
        _, lo, hi = seg
        n_seg = np.clip(np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), n_fil))),
                        lo, hi).astype(np.int32)
    else:
        n_seg = np.full(n_fil, seg, dtype=np.int32)
    if isinstance(w["lp"], tuple):
        _, lo, hi = w["lp"]
        lp = rng.uniform(lo, hi, n_fil)
    else:
        lp = np.full(n_fil, w["lp"])
    lengths = n_seg.astype(np.float64)  # bond length 1
    insert = insert or _library_insert
    sites = insert(w["n_dim"], 0.5 * side, seed, n_seg, lengths, lp,
                   diameter=DIAMETER, insertion=w.get("insertion", "random"))
    system = dict(n_dim=w["n_dim"], system_radius=0.5 * side, delta=w["delta"],
                  wca_eps=1.0, wca_sig=1.0, f_cutoff=2000.0,
                  stoch_flag=1 if stoch else 0, interaction_flag=1 if interaction else 0,
                  like_like_interactions=1, seed=seed if precision_seed is None else precision_seed)
    filaments = [dict(length=float(lengths[i]), persistence_length=float(lp[i]),
                      diameter=DIAMETER, min_bond_length=MIN_BOND_LENGTH,
                      friction_ratio=FRICTION_RATIO) for i in range(n_fil)]
    return system, filaments, sites
