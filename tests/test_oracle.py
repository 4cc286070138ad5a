"""CPU oracle: pinned against the reference's own code.

* Philox4x32-10 against the published known-answer vectors (Salmon et al.).
* The oracle replays the golden fixtures of tests/golden/ -- generated by
  tests/golden/make_golden.py from the reference's own sources
  (oracle/_ref) -- bit for bit, including rebuilds and renormalisations,
  and the pressure records and potential energies of the thermo_* ones.
* Where the reference build is present, both run side by side on a fresh
  configuration and must agree bit for bit every step.
* Analytic known answers: WCA force of two segments at a known distance and
  its cap; a straight rod without noise or forces does not move.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

from checkers import Oracle, Reference, ORACLE_SO, SystemDesc

_ALL_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
GOLDEN = [p for p in _ALL_GOLDEN if os.path.basename(p).startswith("ref")]
THERMO_GOLDEN = [p for p in _ALL_GOLDEN if os.path.basename(p).startswith("thermo_")]


def _oracle_lib():
    return ctypes.CDLL(ORACLE_SO)


def test_philox_known_answers():
    lib = _oracle_lib()
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kat:
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        o = (ctypes.c_uint32 * 4)()
        lib.sco_philox4x32_10(c, k, o)
        assert tuple(o) == want


def _case(path):
    z = np.load(path)
    n_dim, R, delta, seed, lp, n_seg, n_fil, steps = z["system"]
    system = dict(n_dim=int(n_dim), system_radius=R, delta=delta, wca_eps=1.0, wca_sig=1.0,
                  f_cutoff=2000.0, stoch_flag=1, interaction_flag=1, like_like_interactions=1,
                  seed=int(seed))
    fils = [dict(length=float(n_seg), persistence_length=float(lp), diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * int(n_fil)
    return z, system, fils, int(steps)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_reference_fixture(path):
    z, system, fils, steps = _case(path)
    nd = system["n_dim"]
    o = Oracle(system, fils, z["sites0"])
    o.step(steps)
    f, t = o.bond_forces()
    sw, nn = o.filament_state()
    checks = {
        "sites": (o.sites()[:, :nd], z["sites"][:, :nd]),
        "prev_sites": (o.prev_sites()[:, :nd], z["prev_sites"][:, :nd]),
        "random_forces": (o.random_forces()[:, :nd], z["random_forces"][:, :nd]),
        "site_forces": (o.site_forces()[:, :nd], z["site_forces"][:, :nd]),
        "bond_force": (f[:, :nd], z["bond_force"][:, :nd]),
        "bond_torque": (t, z["bond_torque"]),
        "tensions": (o.tensions(), z["tensions"]),
        "pairs": (o.pairs(), z["pairs"]),
        "dr_tot": (o.dr_tot(), z["dr_tot"]),
        "normalize_switch": (sw, z["normalize_switch"]),
        "n_normalize": (nn, z["n_normalize"]),
        "bond_cells": (o.bond_cells(), z["bond_cells"]),
    }
    for name, (a, b) in checks.items():
        assert a.shape == b.shape, name
        assert np.array_equal(a, b), name
    assert o.n_rebuilds == int(z["n_rebuilds"][0])
    assert o.n_rebuilds > 0


@pytest.mark.parametrize("path", THERMO_GOLDEN, ids=[os.path.basename(p) for p in THERMO_GOLDEN])
def test_oracle_reproduces_reference_thermo_fixture(path):
    """Pressure records every n_thermo steps, the running virial sum and every
    filament's potential energy, from the reference's own code over a run
    with rebuilds: the oracle gives the same bits."""
    z, system, fils, steps = _case(path)
    o = Oracle(system, fils, z["sites0"])
    o.set_thermo(int(z["n_thermo"][0]))
    o.step(steps)
    st, P, p, V = o.thermo_records()
    assert len(st) == steps // int(z["n_thermo"][0]) == len(z["thermo_step"])
    assert np.array_equal(st, z["thermo_step"])
    assert np.array_equal(P, z["thermo_tensor"])
    assert np.array_equal(p, z["thermo_pressure"])
    assert np.array_equal(V, z["thermo_volume"])
    assert np.array_equal(o.stress(), z["stress"])
    assert np.array_equal(o.potential_energy(), z["potential_energy"])
    assert np.array_equal(o.sites(), z["sites"])
    assert o.n_rebuilds == int(z["n_rebuilds"][0]) > 1
    assert (z["potential_energy"] > 0).any()
    o.close()


def test_fixtures_exercise_rebuilds_and_renormalisation():
    assert len(GOLDEN) >= 3
    for path in GOLDEN:
        z, system, fils, steps = _case(path)
        assert int(z["n_rebuilds"][0]) >= 1
        assert (z["n_normalize"] < steps).any()


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("n_dim", [3, 2])
def test_oracle_and_reference_side_by_side(n_dim):
    import simcore_b200 as sc
    n_fil, n_seg, R = (25, 12, 14.0) if n_dim == 3 else (30, 14, 22.0)
    nb = np.full(n_fil, n_seg, dtype=np.int32)
    sites = sc.insert_filaments(n_dim, R, 99 + n_dim, nb, nb.astype(float), np.full(n_fil, 50.0))
    system = dict(n_dim=n_dim, system_radius=R, delta=2e-4, seed=7)
    fils = [dict(length=float(n_seg), persistence_length=50.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * n_fil
    o = Oracle(system, fils, sites)
    r = Reference(system, fils, sites, n_threads=2)
    for _ in range(30):
        o.step(3)
        r.step(3)
        assert np.array_equal(o.sites()[:, :n_dim], r.sites()[:, :n_dim])
        assert np.array_equal(o.bond_forces()[0][:, :n_dim], r.bond_forces()[0][:, :n_dim])
        assert np.array_equal(o.tensions(), r.tensions())
        assert np.array_equal(o.pairs(), r.pairs())
    assert o.n_rebuilds == r.n_rebuilds


def _segment_force(a1, a2, b1, b2):
    lib = _oracle_lib()
    sysd = SystemDesc(n_dim=3, system_radius=50.0, delta=1e-4, wca_eps=1.0, wca_sig=1.0,
                      f_cutoff=2000.0, stoch_flag=0, interaction_flag=1,
                      like_like_interactions=1, seed=0, n_threads=1)
    arr = lambda v: (ctypes.c_double * 3)(*v)  # noqa: E731
    out = (ctypes.c_double * 3)()
    lib.sco_segment_force.restype = ctypes.c_int
    inside = lib.sco_segment_force(ctypes.byref(sysd), arr(a1), arr(a2), arr(b1), arr(b2), out)
    return inside, np.array(out[:])


def test_wca_known_answers():
    rcut = 2 ** (1 / 6)
    for r in (0.9, 1.0, 1.1):
        inside, f = _segment_force([0, 0, 0], [1, 0, 0], [0, r, 0], [1, r, 0])
        assert inside == 1
        # F = -24 eps (2 sigma^12 / r^13 - sigma^6 / r^7) along y, pushing a away from b
        fa = -24.0 * (2.0 / r ** 13 - 1.0 / r ** 7)
        assert abs(f[1] - fa) <= 1e-12 * abs(fa)
        assert f[0] == 0 and f[2] == 0
    inside, f = _segment_force([0, 0, 0], [1, 0, 0], [0, 0.5, 0], [1, 0.5, 0])
    assert f[1] == -2000.0  # capped at f_cutoff
    inside, f = _segment_force([0, 0, 0], [1, 0, 0], [0, rcut + 0.01, 0], [1, rcut + 0.01, 0])
    assert inside == 0
    # periodic image across the box face (side 100)
    inside, f = _segment_force([-49.8, 0, 0], [-49.8, 1, 0], [49.2, 0, 0], [49.2, 1, 0])
    assert inside == 1 and f[0] > 0


def _straight_rod(interaction):
    n_seg = 10
    sites = np.zeros((n_seg + 1, 3))
    sites[:, 0] = np.arange(n_seg + 1) - 5.0
    system = dict(n_dim=3, system_radius=20.0, delta=1e-3, stoch_flag=0, seed=0,
                  interaction_flag=interaction)
    fils = [dict(length=float(n_seg), persistence_length=100.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)]
    return Oracle(system, fils, sites), sites


def test_straight_rod_without_noise_or_interactions_stays_put():
    o, sites = _straight_rod(0)
    o.step(20)
    assert np.allclose(o.sites(), sites, atol=1e-12)
    assert np.abs(o.tensions()).max() < 1e-9


def test_straight_rod_second_neighbour_bonds_repel():
    """Bonds i and i+2 of one filament are not excluded (only bonds sharing a
    site are, reference src/bond.cpp:118-121); on a straight rod with unit
    bonds they are 1 sigma apart, inside the WCA cutoff, so candidate pairs
    among them push with 24 eps/sigma and the tensions balance the push: the
    rod does not move."""
    o, sites = _straight_rod(1)
    o.step(1)
    f, _ = o.bond_forces()
    assert np.allclose(np.abs(f[:, 0][f[:, 0] != 0]), 24.0)
    assert np.abs(o.tensions()).max() > 1.0
    o.step(19)
    assert np.allclose(o.sites(), sites, atol=1e-12)


def _two_rods(n_dim, gap):
    """Two straight 5-bond rods along x, `gap` apart in y, no noise."""
    sites = np.zeros((12, 3))
    sites[:6, 0] = np.arange(6) - 2.5
    sites[6:, 0] = np.arange(6) - 2.5
    sites[6:, 1] = gap
    system = dict(n_dim=n_dim, system_radius=10.0, delta=1e-4, stoch_flag=0, seed=0,
                  interaction_flag=1)
    fils = [dict(length=5.0, persistence_length=100.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * 2
    return system, fils, sites


@pytest.mark.parametrize("n_dim", [2, 3])
def test_crosslink_tether_known_answer(n_dim):
    """Two tethers (k 10, rest 1) between rods 1.5 apart (beyond the WCA
    cutoff): tail-to-tail on bond 0 of each rod and head-to-head on the last
    bonds.  Step 1 (odd) applies the zero forces stored so far; step 2 (even)
    computes F = k (|dr| - rest) = 5 along +y on anchor 0, -F on anchor 1, and
    torques (lambda - l/2) u x F = -/+2.5 z at the tails, +/-2.5 z at the
    heads (src/crosslink.cpp:247-275, src/anchor.cpp:132-146)."""
    system, fils, sites = _two_rods(n_dim, 1.5)
    o = Oracle(system, fils, sites)
    o.add_crosslinks([0, 5], [6, 11], k_spring=10.0, rest_length=1.0)
    o.step(1)
    f, t = o.bond_forces()
    assert np.all(f == 0) and np.all(t == 0)
    assert np.all(o.crosslink_forces() == 0)
    o.step(1)
    xf = o.crosslink_forces()
    assert np.allclose(xf, [[0, 5, 0], [0, 5, 0]], atol=1e-12)
    f, t = o.bond_forces()
    assert np.allclose(f[0], [0, 5, 0]) and np.allclose(f[5], [0, -5, 0])
    assert np.allclose(f[4], [0, 5, 0]) and np.allclose(f[9], [0, -5, 0])
    assert np.allclose(t[0], [0, 0, -2.5]) and np.allclose(t[5], [0, 0, 2.5])
    assert np.allclose(t[4], [0, 0, 2.5]) and np.allclose(t[9], [0, 0, -2.5])
    assert np.all(f[[1, 2, 3, 6, 7, 8]] == 0)
    # Step 3 (odd) re-applies the step-2 forces unchanged although the rods
    # have moved.
    before = o.sites()
    o.step(1)
    assert not np.array_equal(o.sites(), before)
    f3, t3 = o.bond_forces()
    assert np.array_equal(f3, f) and np.array_equal(t3, t)
    # The tether pulls the rods together.
    assert o.sites()[6:, 1].mean() < 1.5 and o.sites()[:6, 1].mean() > 0.0


def test_crosslink_compression_constant():
    """k_spring_compress >= 0 replaces k_spring when the tether is shorter
    than its rest length."""
    system, fils, sites = _two_rods(3, 1.5)
    o = Oracle(system, fils, sites)
    o.add_crosslinks([0], [6], k_spring=10.0, k_spring_compress=4.0, rest_length=2.0)
    o.step(2)
    assert np.allclose(o.crosslink_forces(), [[0, -2.0, 0]], atol=1e-12)


def _mean_bond_cosine(xyz, n_sites):
    off = np.concatenate([[0], np.cumsum(n_sites)])
    cos = []
    for f in range(len(n_sites)):
        u = np.diff(xyz[off[f]:off[f + 1]], axis=0)
        u /= np.linalg.norm(u, axis=1)[:, None]
        cos.append((u[1:] * u[:-1]).sum(1))
    return float(np.concatenate(cos).mean())


@pytest.mark.parametrize("lp,dt,stable", [(500.0, 1e-4, True), (1000.0, 1e-4, False),
                                          (1000.0, 5e-5, True)])
def test_explicit_bending_stability_limit(lp, dt, stable):
    """The reference's bending forces are explicit, so with 1-sigma bonds its
    midpoint step is stable only below a persistence length set by dt:
    20 filaments of 50 bonds, no pair forces, 400 steps.  At workload E's
    lp 1000 and dt 1e-4 the filaments buckle (mean bond cosine about 0.72
    against the worm-like-chain 0.999); at lp 500, or at dt 5e-5, they stay
    within 1e-3 of it."""
    import simcore_b200 as sc
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("E", 0.002, seed=1)
    fils = [dict(f, persistence_length=lp) for f in fils]
    o = Oracle(dict(system, interaction_flag=0, delta=dt), fils, sites)
    o.step(400)
    n_sites = np.array([sc.filament_n_bonds(f) + 1 for f in fils])
    c = _mean_bond_cosine(o.sites(), n_sites)
    o.close()
    wlc = 1.0 / np.tanh(lp) - 1.0 / lp
    if stable:
        assert abs(c - wlc) < 1e-3, (c, wlc)
    else:
        assert c < 0.9, (c, wlc)


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
@pytest.mark.parametrize("n_dim", [3, 2])
def test_thermo_and_potentials_match_reference(n_dim):
    """The pair virial the reference sums every step (ApplyPairInteractions),
    its pressure records every n_thermo steps (CalculatePressure, with the
    Space's volume and the interactor count) and every filament's potential
    energy: oracle and the reference's own code bit for bit, over runs with
    rebuilds."""
    import simcore_b200 as sc
    n_fil, n_seg, R = (25, 12, 14.0) if n_dim == 3 else (30, 14, 22.0)
    nb = np.full(n_fil, n_seg, dtype=np.int32)
    sites = sc.insert_filaments(n_dim, R, 99 + n_dim, nb, nb.astype(float), np.full(n_fil, 50.0))
    system = dict(n_dim=n_dim, system_radius=R, delta=2e-4, seed=7)
    fils = [dict(length=float(n_seg), persistence_length=50.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * n_fil
    o = Oracle(system, fils, sites)
    r = Reference(system, fils, sites, n_threads=2)
    o.set_thermo(6)
    r.set_thermo(6)
    n_rec = 0
    for _ in range(10):
        o.step(9)
        r.step(9)
        a, b = o.thermo_records(), r.thermo_records()
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        n_rec += len(a[0])
        assert np.array_equal(o.stress(), r.stress())
        assert np.array_equal(o.potential_energy(), r.potential_energy())
    assert n_rec == 90 // 6 and o.n_rebuilds > 1
    assert (o.potential_energy() > 0).any()
    o.close()
    r.close()


def test_ideal_pressure_without_contacts():
    """Two two-bond rods (bond length 3, so a rod's only bond pair is
    adjacent and excluded) far apart, no noise: no pair is in range, so the
    pressure tensor is the ideal n_bonds / V on the diagonal and the
    potentials are zero."""
    import simcore_b200 as sc
    R = 20.0
    fils = [dict(length=6.0, persistence_length=100.0, diameter=1.0, min_bond_length=2.0,
                 friction_ratio=2.0)] * 2
    assert sc.filament_n_bonds(fils[0]) == 2
    sites = np.zeros((6, 3))
    sites[:3, 0] = [-3.0, 0.0, 3.0]
    sites[3:, 0] = [-3.0, 0.0, 3.0]
    sites[3:, 1] = 10.0
    system = dict(n_dim=3, system_radius=R, delta=1e-4, seed=1, stoch_flag=0)
    o = Oracle(system, fils, sites)
    o.set_thermo(2)
    o.step(4)
    st, P, p, V = o.thermo_records()
    assert list(st) == [2, 4]
    ideal = 4 * (1.0 / (2 * R) ** 3)
    assert np.array_equal(V, np.full(2, (2 * R) ** 3))
    assert np.array_equal(P[:, [0, 4, 8]], np.full((2, 3), ideal))
    assert not P[:, [1, 2, 3, 5, 6, 7]].any()
    assert np.array_equal(p, np.full(2, (ideal + ideal + ideal) / 3))
    assert not o.potential_energy().any()
    o.close()


@pytest.mark.parametrize("name,scale", [("A", 1.0), ("B", 0.05), ("C", 0.004), ("E", 0.02)])
def test_oracle_insertion_is_the_library_insertion(name, scale):
    """The oracle's insertion (restated from the reference's distributions,
    the shared Philox insertion stream and the longest-first order) gives
    the library's host insertion bit for bit, so a CPU run of the reference's
    code can start from the GPU run's configuration without loading the CUDA
    library."""
    import simcore_b200  # noqa: F401  (host insertion; no device needed)
    from simcore_b200 import workloads
    from checkers import oracle_insert, workloads_module
    lib_sites = workloads.make(name, scale, seed=3)[2]
    orc_sites = workloads_module().make(name, scale, seed=3, insert=oracle_insert)[2]
    assert np.array_equal(lib_sites, orc_sites)


def test_oracle_insertion_of_replica_batches():
    from simcore_b200 import workloads
    from checkers import oracle_insert, workloads_module
    a = workloads.make_replicas("D", n_replicas=3, fil_scale=0.2, seed=5)
    b = workloads_module().make_replicas("D", n_replicas=3, fil_scale=0.2, seed=5,
                                         insert=oracle_insert)
    assert np.array_equal(a[2], b[2])
    assert a[3] == b[3]


TETHER_GOLDEN = [p for p in _ALL_GOLDEN if os.path.basename(p).startswith("tether_")]


@pytest.mark.parametrize("path", TETHER_GOLDEN, ids=os.path.basename)
def test_oracle_reproduces_reference_tether_fixture(path):
    """Doubly-bound crosslinks as the reference's own Crosslink and Anchor
    code runs them (tests/golden/make_golden.py, tether_* fixtures): anchors
    keep their mesh lambda while the bonds stretch, move between neighbouring
    bonds, and apply their tether forces on even steps and again on odd
    ones.  The oracle reproduces positions, bond forces and torques, tensions
    and tether forces bit for bit."""
    g = np.load(path)
    nd, R, delta, seed, lp, nseg, nfil, steps = g["system"]
    k, kc, rest = g["links"]
    system = dict(n_dim=int(nd), system_radius=R, delta=delta, seed=int(seed))
    fils = [dict(length=float(nseg), persistence_length=lp, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * int(nfil)
    o = Oracle(system, fils, g["sites0"])
    o.add_crosslinks(g["site_a"], g["site_b"], k_spring=k, k_spring_compress=kc,
                     rest_length=rest)
    o.step(int(steps))
    f, t = o.bond_forces()
    for name, got in (("sites", o.sites()), ("prev_sites", o.prev_sites()),
                      ("bond_force", f), ("bond_torque", t), ("tensions", o.tensions()),
                      ("crosslink_forces", o.crosslink_forces())):
        assert np.array_equal(got, g[name]), name
    assert o.n_rebuilds == int(g["n_rebuilds"][0])
    o.close()


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
def test_oracle_and_reference_tethers_side_by_side():
    """A tethered network of buckling filaments (workload E's parameters at
    small size), the oracle and the reference's own code stepped together:
    equal bits every step."""
    from checkers import oracle_insert, oracle_n_bonds, workloads_module
    wl = workloads_module()
    system, fils, sites = wl.make("E", 0.01, seed=4, insert=oracle_insert)
    a, b, k, rest = wl.crosslinks("E", sites, fils, 2 * system["system_radius"], scale=0.01,
                                  seed=4, n_bonds=oracle_n_bonds)
    o = Oracle(system, fils, sites)
    r = Reference(system, fils, sites)
    for c in (o, r):
        c.add_crosslinks(a, b, k_spring=k, rest_length=rest)
    for _ in range(12):
        o.step(1)
        r.step(1)
        assert np.array_equal(o.crosslink_forces(), r.crosslink_forces())
        assert np.array_equal(o.bond_forces()[0], r.bond_forces()[0])
        assert np.array_equal(o.sites(), r.sites())
    o.close()
    r.close()


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
def test_reference_analysis_hooks_run():
    """The checker's analysis hooks (the reference's RunMse2eAnalysis /
    RunThetaAnalysis and diffusion analysis on its own filaments) give a
    mean-square end-to-end distance below L^2, one histogram count per joint
    and filament, and finite diffusion means."""
    from checkers import oracle_insert
    nb = np.full(10, 12, dtype=np.int32)
    sites = oracle_insert(3, 12.0, 3, nb, nb.astype(float), np.full(10, 20.0))
    system = dict(n_dim=3, system_radius=12.0, delta=2e-4, seed=3)
    fils = [dict(length=12.0, persistence_length=20.0, diameter=1.0, min_bond_length=0.666,
                 friction_ratio=2.0)] * 10
    r = Reference(system, fils, sites)
    r.diffusion_init(3)
    for _ in range(6):
        r.step(4)
        r.analysis_sample(20)
        r.diffusion_sample()
    m, e, n, hist = r.analysis_results()
    assert 0 < m < 144.0 and e > 0 and n == 6
    assert hist.shape == (11, 20) and hist.sum() == 6 * 10 * 11
    for a in r.diffusion_results():
        assert np.all(np.isfinite(a))
    r.close()
