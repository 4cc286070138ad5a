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
  E  10,000 x 50 bonds, lp 1000, side 150, dt 1e-4      (network geometry)

scale < 1 shrinks the filament count and the box volume together (same
density) for parity tests at small sizes.
"""
import math

import numpy as np

from . import insert_filaments

MIN_BOND_LENGTH = 0.666
DIAMETER = 1.0
FRICTION_RATIO = 2.0

WORKLOADS = {
    "A": dict(n_dim=3, side=50.0, n_fil=100, n_seg=20, lp=500.0, delta=1e-4, n_steps=1000),
    "B": dict(n_dim=3, side=200.0, n_fil=20000, n_seg=10, lp=100.0, delta=1e-4, n_steps=2000),
    "C": dict(n_dim=3, side=300.0, n_fil=50000, n_seg=("loguniform", 5, 200),
              lp=("uniform", 10.0, 1000.0), delta=5e-5, n_steps=1000),
    "E": dict(n_dim=3, side=150.0, n_fil=10000, n_seg=50, lp=1000.0, delta=1e-4, n_steps=1000),
}


def describe(name):
    w = WORKLOADS[name]
    return dict(w)


def make(name, scale=1.0, seed=0, precision_seed=None, stoch=True, interaction=True):
    """Returns (system, filaments, sites) for workload `name`."""
    w = WORKLOADS[name]
    n_fil = max(2, int(round(w["n_fil"] * scale)))
    side = w["side"] * (scale ** (1.0 / w["n_dim"]))
    rng = np.random.default_rng(seed + 12345)
    if isinstance(w["n_seg"], tuple):
        _, lo, hi = w["n_seg"]
        n_seg = np.clip(np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), n_fil))),
                        lo, hi).astype(np.int32)
    else:
        n_seg = np.full(n_fil, w["n_seg"], dtype=np.int32)
    if isinstance(w["lp"], tuple):
        _, lo, hi = w["lp"]
        lp = rng.uniform(lo, hi, n_fil)
    else:
        lp = np.full(n_fil, w["lp"])
    lengths = n_seg.astype(np.float64)  # bond length 1
    sites = insert_filaments(w["n_dim"], 0.5 * side, seed, n_seg, lengths, lp,
                             diameter=DIAMETER)
    system = dict(n_dim=w["n_dim"], system_radius=0.5 * side, delta=w["delta"],
                  wca_eps=1.0, wca_sig=1.0, f_cutoff=2000.0,
                  stoch_flag=1 if stoch else 0, interaction_flag=1 if interaction else 0,
                  like_like_interactions=1, seed=seed if precision_seed is None else precision_seed)
    filaments = [dict(length=float(lengths[i]), persistence_length=float(lp[i]),
                      diameter=DIAMETER, min_bond_length=MIN_BOND_LENGTH,
                      friction_ratio=FRICTION_RATIO) for i in range(n_fil)]
    return system, filaments, sites
