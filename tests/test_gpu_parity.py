"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

The FP64 path is bit-identical to the oracle (which is itself bit-identical
to the reference's own code, see test_oracle.py): every comparison below is
exact equality, over single steps and over long runs that include pair-list
rebuilds and bond renormalisations.
"""
import numpy as np
import pytest

from checkers import Oracle

pytestmark = pytest.mark.gpu


def _ctx(system, filaments, sites, precision="fp64"):
    import simcore_b200 as sc
    return sc.Context(system, filaments, sites, precision=precision)


def _workload(name, scale, seed=0, **kw):
    from simcore_b200 import workloads
    return workloads.make(name, scale=scale, seed=seed, **kw)


def assert_same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, what
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if bad.any():
        idx = np.argwhere(bad)[0]
        raise AssertionError("%s differs at %s: %r vs %r (%d entries)"
                             % (what, idx, a[tuple(idx)], b[tuple(idx)], bad.sum()))


def compare_state(ctx, o, nd, capture=True):
    assert_same(ctx.sites()[:, :nd], o.sites()[:, :nd], "sites")
    assert_same(ctx.prev_sites()[:, :nd], o.prev_sites()[:, :nd], "prev sites")
    assert_same(ctx.random_forces()[:, :nd], o.random_forces()[:, :nd], "random forces")
    gf, gt = ctx.bond_forces()
    of, ot = o.bond_forces()
    assert_same(gf[:, :nd], of[:, :nd], "bond forces")
    assert_same(gt, ot, "bond torques")
    if capture:
        assert_same(ctx.site_forces()[:, :nd], o.site_forces()[:, :nd], "site forces")
        assert_same(ctx.tensions(), o.tensions(), "tensions")
    assert_same(ctx.pairs(), o.pairs(), "pair list")
    if o.i_step % 2 == 1:
        # The GPU adds a full step's displacement in that step's epilogue;
        # the reference adds it at the next (odd) step's rebuild check.  The
        # two agree whenever that check has happened, i.e. after odd steps.
        assert_same(ctx.dr_tot(), o.dr_tot(), "dr_tot")
    sw, nn = ctx.filament_state()
    osw, onn = o.filament_state()
    assert_same(sw, osw, "normalize_switch")
    assert_same(nn, onn, "n_normalize")
    assert ctx.counters().n_rebuilds == o.n_rebuilds


@pytest.mark.parametrize("fused", [True, False])
def test_fp64_single_steps_bitwise(fused):
    system, fils, sites = _workload("A", 0.3, seed=3)
    ctx = _ctx(system, fils, sites)
    ctx.set_capture(True)
    o = Oracle(system, fils, sites)
    assert_same(ctx.pairs(), o.pairs(), "initial pair list (before culling both drop exclusions)")
    for _ in range(7):
        if fused:
            ctx.step(1)
        else:
            ctx.interact()
            ctx.update_positions()
        o.step(1)
        compare_state(ctx, o, 3)


def test_fp64_workload_A_run_bitwise():
    """Full-size workload A (100 x 20 bonds) for 408 steps: identical state,
    identical rebuild count and pair lists, every 51 steps."""
    system, fils, sites = _workload("A", 1.0, seed=0)
    ctx = _ctx(system, fils, sites)
    ctx.set_capture(True)
    o = Oracle(system, fils, sites)
    for _ in range(8):
        ctx.step(51)
        o.step(51)
        compare_state(ctx, o, 3)
    assert o.n_rebuilds > 5


def test_fp64_2d_bitwise():
    import simcore_b200 as sc
    n_fil, n_seg, R = 60, 16, 30.0
    nb = np.full(n_fil, n_seg, dtype=np.int32)
    sites = sc.insert_filaments(2, R, 7, nb, nb.astype(float), np.full(n_fil, 200.0))
    system = dict(n_dim=2, system_radius=R, delta=1e-4, stoch_flag=1, interaction_flag=1,
                  like_like_interactions=1, seed=5)
    fils = [dict(length=float(n_seg), persistence_length=200.0, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * n_fil
    ctx = _ctx(system, fils, sites)
    ctx.set_capture(True)
    o = Oracle(system, fils, sites)
    for _ in range(6):
        ctx.step(41)
        o.step(41)
        compare_state(ctx, o, 2)


def test_bond_cells_and_pairs_bitwise():
    system, fils, sites = _workload("B", 0.05, seed=1)
    ctx = _ctx(system, fils, sites)
    o = Oracle(system, fils, sites)
    assert ctx.counters().n_cells_1d == o.n_cells_1d
    assert_same(ctx.bond_cells(), o.bond_cells(), "bond cells")
    ctx.step(1)
    o.step(1)
    assert_same(ctx.pairs(), o.pairs(), "pair list")


def test_mixed_force_error():
    """Mixed precision (FP32 pair forces) against FP64 on the same state:
    max |dF| / max |F| <= 1e-5 over all bond forces and torques."""
    system, fils, sites = _workload("B", 0.1, seed=2)
    c64 = _ctx(system, fils, sites, "fp64")
    c32 = _ctx(system, fils, sites, "mixed")
    c64.interact()
    c32.interact()
    f64, t64 = c64.bond_forces()
    f32, t32 = c32.bond_forces()
    ef = np.abs(f32 - f64).max() / np.abs(f64).max()
    et = np.abs(t32 - t64).max() / np.abs(t64).max()
    assert ef <= 1e-5, ef
    assert et <= 1e-5, et


@pytest.mark.parametrize("angle", [0.0, 3e-5, 1.7e-4, 2e-3, 5e-3])
def test_mixed_near_parallel_pairs(angle):
    """Two straight rods side by side 1.05 apart (inside the WCA range),
    overlapping, at a small angle.  Within about 0.2 degrees of parallel,
    FP32's 1 - c^2 is rounding alone and the closest points it finds can be
    far off; the default mixed pair stage evaluates those pairs from the
    FP64 sites (exactly parallel rods and wider angles stay in FP32).
    Forces and torques then match the FP64 path to 1e-5 of the largest at
    every angle."""
    R = 20.0
    j = np.arange(11.0)
    sites = np.zeros((22, 3))
    sites[:11, 0] = j - 5.0
    sites[11:, 0] = -4.7 + j * np.cos(angle)
    sites[11:, 2] = 1.05 + j * np.sin(angle)
    system = dict(n_dim=3, system_radius=R, delta=1e-4, seed=1, stoch_flag=0)
    fils = [dict(length=10.0, persistence_length=100.0, diameter=1.0, min_bond_length=0.666,
                 friction_ratio=2.0)] * 2
    c64 = _ctx(system, fils, sites, "fp64")
    c32 = _ctx(system, fils, sites, "mixed")
    assert len(c64.pairs()) > 0
    for c in (c64, c32):
        c.interact()
    f64, t64 = c64.bond_forces()
    f32, t32 = c32.bond_forces()
    assert np.abs(f64).max() > 1.0
    assert np.abs(f32 - f64).max() <= 1e-5 * np.abs(f64).max()
    assert np.abs(t32 - t64).max() <= 1e-5 * max(np.abs(t64).max(), np.abs(f64).max())


def test_exact_near_parallel_graph_matches_host():
    """The captured graph, whose pair kernels evaluate nearly parallel pairs
    from the FP64 sites in their last block, gives the host-driven loop's
    bits, on a batch of independent 2D systems."""
    system, fils, sites, reps = _replica_batch(3, 0.05, seed=4)
    a = _ctx_replicas(system, fils, sites, reps, "mixed")
    b = _ctx_replicas(system, fils, sites, reps, "mixed")
    a.step_graph(40)
    b.step(40)
    assert_same(a.sites(), b.sites(), "sites")
    assert a.counters().n_rebuilds == b.counters().n_rebuilds


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_path_matches_host_path(precision):
    """The captured WHILE-loop graph (device-decided rebuilds) gives the same
    bits as the host-driven loop, in both precisions."""
    system, fils, sites = _workload("B", 0.05, seed=6)
    a = _ctx(system, fils, sites, precision)
    b = _ctx(system, fils, sites, precision)
    for n in (40, 41, 20):
        a.step_graph(n)
        b.step(n)
        assert_same(a.sites(), b.sites(), "sites")
        assert_same(a.pairs(), b.pairs(), "pairs")
        assert a.counters().n_rebuilds == b.counters().n_rebuilds
    assert a.counters().n_rebuilds > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_captured_run_grows_an_overflowing_pair_list(precision):
    """Stiff filaments (persistence length 1000 at dt 1e-4, 50 bonds) buckle
    under the reference's explicit bending, and their candidate pairs grow
    about fivefold in 400 steps: past the half-again headroom a captured run
    starts with.  The run stops at the overflowing rebuild, grows the list,
    redoes the rebuild and resumes -- bit for bit the host-driven run, with
    the same rebuild count."""
    system, fils, sites = _workload("E", 0.1, seed=3)
    a = _ctx(system, fils, sites, precision)
    b = _ctx(system, fils, sites, precision)
    n0 = a.counters().n_pairs
    a.step_graph(400)
    b.step(400)
    ca, cb = a.counters(), b.counters()
    assert ca.n_list_regrowths > 0
    assert ca.n_pairs > 2 * n0
    assert ca.i_step == cb.i_step == 400
    assert ca.n_rebuilds == cb.n_rebuilds
    assert_same(a.sites(), b.sites(), "sites")
    assert_same(a.pairs(), b.pairs(), "pairs")
    a.close()
    b.close()


def test_graph_matches_oracle():
    system, fils, sites = _workload("A", 1.0, seed=4)
    ctx = _ctx(system, fils, sites)
    o = Oracle(system, fils, sites)
    for _ in range(3):
        ctx.step_graph(101)
        o.step(101)
        compare_state(ctx, o, 3, capture=False)


def _fast_vs_exact(system, fils, sites):
    """One BD step of the fast and the exact integrator on identical forces:
    without noise, positions agree to 1e-12 relative (FMA contraction,
    reciprocals, two-sided or parallel-cyclic solves: FP64 rounding only);
    with noise, which the fast step draws and projects in FP32, the
    displacements agree to 1e-6 of the largest one (the FP32 uniforms are
    within 2^-24 of the FP64 ones)."""
    quiet = dict(system, stoch_flag=0)
    a = _ctx(quiet, fils, sites, "mixed")
    b = _ctx(quiet, fils, sites, "mixed")
    b.set_fast_integrator(False)
    a.step(2)
    b.step(2)
    ra, rb = a.sites(), b.sites()
    assert np.abs(ra - rb).max() <= 1e-12 * np.abs(rb).max()
    a = _ctx(system, fils, sites, "mixed")
    b = _ctx(system, fils, sites, "mixed")
    b.set_fast_integrator(False)
    a.step(2)
    b.step(2)
    ra, rb = a.sites(), b.sites()
    disp = np.abs(rb - sites).max()
    assert disp > 0
    assert np.abs(ra - rb).max() <= 1e-6 * disp
    return a, b


def test_fast_integrator_long_filaments_close_to_exact():
    """Workload C's length spread (5 to 200 bonds): the fast integrator solves
    the 256-site blocks that hold a filament of more than 32 bonds by
    parallel cyclic reduction.  Against the exact integrator (the
    reference's sequential Thomas) on identical forces: see _fast_vs_exact;
    the captured run gives the host-driven loop's bits."""
    system, fils, sites = _workload("C", 0.002, seed=3, side=150.0)
    assert max(f["length"] for f in fils) > 128
    _fast_vs_exact(system, fils, sites)
    c = _ctx(system, fils, sites, "mixed")
    d = _ctx(system, fils, sites, "mixed")
    c.step_graph(40)
    d.step(40)
    assert_same(c.sites(), d.sites(), "sites")


def test_fast_integrator_close_to_exact():
    """The mixed path's fast integrator against the exact FP64 integrator on
    identical forces (both mixed precision): see _fast_vs_exact."""
    system, fils, sites = _workload("B", 0.05, seed=8)
    _fast_vs_exact(system, fils, sites)


def _workload_E(scale, seed=0):
    """Workload E's density, stiffness and tethers, with 10-bond filaments so
    that a small box holds them."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("E", scale=scale, seed=seed, n_seg=10)
    a, b, k, rest = workloads.crosslinks("E", sites, fils, 2 * system["system_radius"],
                                         scale=scale, seed=seed)
    return system, fils, sites, (a, b, k, rest)


def test_crosslinks_fp64_bitwise():
    """Workload E at 1/100 scale (100 x 10 bonds, up to 1,000 tethers): the
    tether kernel, the per-bond anchor sums and the stale odd-step forces are
    bit-identical to the oracle, host-driven and through the captured graph."""
    system, fils, sites, (a, b, k, rest) = _workload_E(0.01, seed=4)
    ctx = _ctx(system, fils, sites)
    ctx.set_capture(True)
    o = Oracle(system, fils, sites)
    ctx.add_crosslinks(a, b, k_spring=k, rest_length=rest)
    o.add_crosslinks(a, b, k_spring=k, rest_length=rest)
    for _ in range(4):
        ctx.step(1)
        o.step(1)
        compare_state(ctx, o, 3)
        assert_same(ctx.crosslink_forces(), o.crosslink_forces(), "tether forces")
    assert np.abs(o.crosslink_forces()).max() > 0
    ctx.set_capture(False)
    for n in (41, 60):
        ctx.step_graph(n)
        o.step(n)
        compare_state(ctx, o, 3, capture=False)
        assert_same(ctx.crosslink_forces(), o.crosslink_forces(), "tether forces")


def test_crosslinks_mixed_close():
    """Mixed precision with tethers, one step after identical starts: bond
    forces (FP64 tethers plus FP32 pair sums) and tether forces within 1e-5
    (relative to the largest) of the FP64 path."""
    system, fils, sites, (a, b, k, rest) = _workload_E(0.01, seed=5)
    c64 = _ctx(system, fils, sites, "fp64")
    c32 = _ctx(system, fils, sites, "mixed")
    for c in (c64, c32):
        c.add_crosslinks(a, b, k_spring=k, rest_length=rest)
        c.step(1)
        c.interact()
    f64, t64 = c64.bond_forces()
    f32, t32 = c32.bond_forces()
    assert np.abs(f32 - f64).max() / np.abs(f64).max() <= 1e-5
    assert np.abs(t32 - t64).max() / np.abs(t64).max() <= 1e-5
    x32, x64 = c32.crosslink_forces(), c64.crosslink_forces()
    assert np.abs(x32 - x64).max() <= 1e-5 * np.abs(x64).max()


@pytest.mark.parametrize("name", ["tether_3d", "tether_2d"])
def test_crosslinks_match_reference_fixture(name):
    """Doubly-bound crosslinks run by the reference's own Crosslink and
    Anchor code (tests/golden/make_golden.py, tether_* fixtures): anchors
    follow their mesh lambda and move between neighbouring bonds as the
    bonds stretch.  The FP64 GPU path, host-driven and through the captured
    graph, gives the reference's bits."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    nd, R, delta, seed, lp, nseg, nfil, steps = g["system"]
    k, kc, rest = g["links"]
    system = dict(n_dim=int(nd), system_radius=R, delta=delta, seed=int(seed))
    fils = [dict(length=float(nseg), persistence_length=lp, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * int(nfil)
    for graph in (False, True):
        ctx = _ctx(system, fils, g["sites0"])
        ctx.add_crosslinks(g["site_a"], g["site_b"], k_spring=k, k_spring_compress=kc,
                           rest_length=rest)
        (ctx.step_graph if graph else ctx.step)(int(steps))
        f, t = ctx.bond_forces()
        nd = int(nd)
        assert_same(ctx.sites()[:, :nd], g["sites"][:, :nd], "sites")
        assert_same(ctx.prev_sites()[:, :nd], g["prev_sites"][:, :nd], "prev sites")
        assert_same(f[:, :nd], g["bond_force"][:, :nd], "bond forces")
        assert_same(t, g["bond_torque"], "bond torques")
        assert_same(ctx.crosslink_forces(), g["crosslink_forces"], "tether forces")
        ctx.close()


def test_fp64_filaments_up_to_500_bonds_bitwise():
    """The reference's longest filaments (max_length 500: 500 bonds at
    min_bond_length 0.666) run on 512-site integrator blocks: bit-identical to
    the oracle over host-driven and captured steps, and the mixed path (block
    PCR) close to it."""
    import simcore_b200 as sc
    lengths = [500.0, 420.0, 300.0, 12.0]
    n_bonds = np.array([int(L) for L in lengths], dtype=np.int32)
    fils = [dict(length=L, persistence_length=200.0, diameter=1.0, min_bond_length=0.666,
                 friction_ratio=2.0) for L in lengths]
    assert [sc.filament_n_bonds(f) for f in fils] == list(n_bonds)
    sites = sc.insert_filaments(3, 300.0, 3, n_bonds, np.array(lengths), np.full(4, 200.0))
    system = dict(n_dim=3, system_radius=300.0, delta=1e-4, seed=3)
    ctx = _ctx(system, fils, sites)
    o = Oracle(system, fils, sites)
    ctx.step(3)
    o.step(3)
    compare_state(ctx, o, 3, capture=False)
    ctx.step_graph(40)
    o.step(40)
    assert_same(ctx.sites(), o.sites(), "sites")
    mixed = _ctx(system, fils, sites, "mixed")
    exact = Oracle(system, fils, sites)
    mixed.step(3)
    exact.step(3)
    d, want = mixed.sites() - sites, exact.sites() - sites
    assert np.abs(d - want).max() <= 1e-6 * np.abs(want).max()


def test_fp64_uneven_lengths_bitwise():
    """Workload C's length and stiffness spread (5 to 200 bonds, log-uniform;
    lp uniform in [10, 1000]) on 100 filaments: 256-site integrator blocks
    holding filaments of mixed lengths, bit-identical to the oracle over
    host-driven and captured steps with rebuilds."""
    system, fils, sites = _workload("C", 0.002, seed=3, side=150.0)
    assert max(f["length"] for f in fils) > 128
    ctx = _ctx(system, fils, sites)
    ctx.set_capture(True)
    o = Oracle(system, fils, sites)
    for _ in range(3):
        ctx.step(1)
        o.step(1)
        compare_state(ctx, o, 3)
    ctx.set_capture(False)
    for n in (101, 100):
        ctx.step_graph(n)
        o.step(n)
        compare_state(ctx, o, 3, capture=False)
    assert o.n_rebuilds > 0


@pytest.mark.parametrize("block", [64, 160, 192])
@pytest.mark.parametrize("precision,fast", [("fp64", False), ("mixed", False), ("mixed", True)])
def test_warp_and_block_integrators_agree(precision, fast, block):
    """The warp-synchronous integrator (filaments of at most 32 sites) and the
    block integrator give the same bits where both are exact, and agree in
    the fast mixed variant to 1e-5 of the largest displacement over the run's
    46 steps (contraction choices and the FP32 noise projection's solve
    order differ, by about 1e-7 of the noise each step);
    blocks of 64 sites run the kernel compiled for up to 128, blocks of 160
    and 192 the one compiled for up to 192."""
    system, fils, sites = _workload("B", 0.05, seed=9)
    a = _ctx(system, fils, sites, precision)
    b = _ctx(system, fils, sites, precision)
    b.set_integrator_layout(0, block)
    for c in (a, b):
        c.set_fast_integrator(fast)
        c.set_capture(True)
    for n in (1, 2, 3):
        a.step(n)
        b.step(n)
    for c in (a, b):
        c.set_capture(False)
    a.step_graph(40)
    b.step_graph(40)
    if precision == "fp64" or not fast:
        assert_same(a.sites(), b.sites(), "sites")
        assert_same(a.pairs(), b.pairs(), "pairs")
    else:
        ra, rb = a.sites(), b.sites()
        assert np.abs(ra - rb).max() <= 1e-5 * np.abs(rb - sites).max()


def test_autotune_leaves_state_and_caches(tmp_path):
    """The autotuner times layouts on the live state and restores it: an
    autotuned FP64 context stays bit-identical to an untuned one (every
    layout is exact).  Its choice is cached per shape and read back."""
    system, fils, sites = _workload("B", 0.05, seed=10)
    a = _ctx(system, fils, sites)
    b = _ctx(system, fils, sites)
    a.step(3)
    b.step(3)
    cache = str(tmp_path / "tune.txt")
    lay = a.autotune(cache)
    assert lay[0] in (0, 32)
    for n in (1, 40):
        a.step_graph(n)
        b.step_graph(n)
        assert_same(a.sites(), b.sites(), "sites")
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1
    c = _ctx(system, fils, sites)
    assert c.autotune(cache) == lay
    assert len(open(cache).read().strip().splitlines()) == 1


def _replica_batch(n_replicas, fil_scale, seed):
    from simcore_b200 import workloads
    return workloads.make_replicas("D", n_replicas=n_replicas, fil_scale=fil_scale, seed=seed)


@pytest.mark.parametrize("graph", [False, True])
def test_replicas_bitwise_per_system(graph):
    """Workload D's batching: five independent 2D systems of different sizes
    in one context.  Each system is bit-identical to its own oracle run --
    sites, bond forces, pair list and rebuild count -- although the systems
    rebuild at different steps and every stage runs for all of them in one
    launch."""
    from simcore_b200 import workloads
    system, fils, sites, reps = _replica_batch(5, 0.03, seed=2)
    ctx = _ctx_replicas(system, fils, sites, reps)
    parts = workloads.split_replicas(system, fils, sites, reps)
    oracles = [Oracle(*p) for p in parts]
    independent = False
    for n in (3, 40, 81):
        if graph:
            ctx.step_graph(n)
        else:
            ctx.step(n)
        for o in oracles:
            o.step(n)
        xyz = ctx.sites()
        f, t = ctx.bond_forces()
        pairs = ctx.pairs()
        nreb, npairs = ctx.replica_counters()
        s0 = b0 = p0 = 0
        for r, o in enumerate(oracles):
            ns, nb = o.n_sites, o.n_bonds
            assert_same(xyz[s0:s0 + ns, :2], o.sites()[:, :2], "system %d sites" % r)
            of, ot = o.bond_forces()
            assert_same(f[b0:b0 + nb, :2], of[:, :2], "system %d bond forces" % r)
            assert_same(t[b0:b0 + nb], ot, "system %d bond torques" % r)
            op = o.pairs()
            assert npairs[r] == len(op)
            assert_same(pairs[p0:p0 + len(op)] - b0, op, "system %d pairs" % r)
            assert nreb[r] == o.n_rebuilds, (r, nreb[r], o.n_rebuilds)
            s0 += ns
            b0 += nb
            p0 += len(op)
        independent = independent or len(set(int(x) for x in nreb)) > 1
    assert independent  # at some point the systems had rebuilt different numbers of times


def test_replicas_mixed_match_single_contexts():
    """Mixed precision: a system advanced inside the batch gives the same bits
    as the same system in a context of its own."""
    from simcore_b200 import workloads
    system, fils, sites, reps = _replica_batch(3, 0.03, seed=3)
    ctx = _ctx_replicas(system, fils, sites, reps, "mixed")
    ctx.step_graph(60)
    xyz = ctx.sites()
    s0 = 0
    for part in workloads.split_replicas(system, fils, sites, reps):
        single = _ctx(*part, precision="mixed")
        single.step_graph(60)
        got = single.sites()
        assert_same(xyz[s0:s0 + len(got)], got, "system sites")
        s0 += len(got)


def _ctx_replicas(system, filaments, sites, replicas, precision="fp64"):
    import simcore_b200 as sc
    return sc.Context(system, filaments, sites, precision=precision, replicas=replicas)


def test_checkpoint_restore_continues_bitwise():
    """A checkpoint taken mid-run (after a midstep, with tethers whose stale
    odd-step forces are part of the state) restores into a fresh context of
    the same systems, which then continues bit for bit as the original."""
    system, fils, sites, (a, b, k, rest) = _workload_E(0.01, seed=6)
    for prec in ("fp64", "mixed"):
        ctx = _ctx(system, fils, sites, prec)
        ctx.add_crosslinks(a, b, k_spring=k, rest_length=rest)
        ctx.step(3)
        ctx.step_graph(48)
        blob = ctx.checkpoint()
        ctx.step_graph(61)
        other = _ctx(system, fils, sites, prec)
        other.add_crosslinks(a, b, k_spring=k, rest_length=rest)
        other.restore(blob)
        other.step_graph(61)
        assert_same(other.sites(), ctx.sites(), "sites")
        assert_same(other.prev_sites(), ctx.prev_sites(), "prev sites")
        assert_same(other.pairs(), ctx.pairs(), "pairs")
        assert_same(other.bond_forces()[0], ctx.bond_forces()[0], "bond forces")
        assert_same(other.crosslink_forces(), ctx.crosslink_forces(), "tether forces")
        assert_same(other.dr_tot(), ctx.dr_tot(), "dr_tot")
        assert other.counters().i_step == ctx.counters().i_step
        assert other.counters().n_rebuilds == ctx.counters().n_rebuilds


def test_checkpoint_of_replicas_and_shape_check():
    """Replica batches checkpoint and restore per system; a checkpoint does
    not load into a context of another shape."""
    import simcore_b200 as sc
    system, fils, sites, reps = _replica_batch(3, 0.03, seed=4)
    ctx = _ctx_replicas(system, fils, sites, reps)
    ctx.step_graph(41)
    blob = ctx.checkpoint()
    ctx.step_graph(40)
    other = _ctx_replicas(system, fils, sites, reps)
    other.restore(blob)
    other.step_graph(40)
    assert_same(other.sites(), ctx.sites(), "sites")
    assert (other.replica_counters()[0] == ctx.replica_counters()[0]).all()
    s2, f2, x2 = _workload("A", 0.1, seed=1)
    wrong = _ctx(s2, f2, x2)
    with pytest.raises(sc.ScError):
        wrong.restore(blob)


def _payload_hash(b):
    """The checkpoint's payload hash: 64-bit FNV-1a over 8-byte words, then
    the tail bytes."""
    import numpy as np
    h = 1469598103934665603
    n8 = len(b) // 8 * 8
    for w in np.frombuffer(b[:n8], dtype="<u8"):
        h = ((h ^ int(w)) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    for x in b[n8:]:
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_restore_rejects_corrupted_checkpoints():
    """A restore checks the blob before it changes the context: a changed
    byte fails the payload hash, and a blob whose hash matches but whose pair
    count exceeds its segment fails the index checks.  The context keeps its
    state through both and continues as before."""
    import struct
    import simcore_b200 as sc
    system, fils, sites = _workload("A", 0.1, seed=21)
    a = _ctx(system, fils, sites)
    a.step(5)
    blob = bytearray(a.checkpoint())
    hdr = 96
    assert struct.unpack_from("<q", blob, 80)[0] == len(blob) - hdr  # payload bytes
    assert struct.unpack_from("<Q", blob, 88)[0] == _payload_hash(bytes(blob[hdr:]))
    bad = bytearray(blob)
    bad[len(bad) // 2] ^= 0x40
    with pytest.raises(sc.ScError, match="hash"):
        a.restore(bytes(bad))
    # One system: the pair count follows the capacity (int32), 13 site arrays
    # of doubles, two filament int arrays and the displacement maxima.
    ns, nf = a.n_sites, a.n_fil
    cap = struct.unpack_from("<i", blob, hdr)[0]
    off_np = hdr + 4 + 13 * 8 * ns + 8 * nf + 8
    assert 0 < struct.unpack_from("<i", blob, off_np)[0] <= cap
    bad = bytearray(blob)
    struct.pack_into("<i", bad, off_np, cap + 1)
    struct.pack_into("<Q", bad, 88, _payload_hash(bytes(bad[hdr:])))
    with pytest.raises(sc.ScError, match="pairs"):
        a.restore(bytes(bad))
    b = _ctx(system, fils, sites)
    b.step(5)
    a.step(7)
    b.step(7)
    assert_same(a.sites(), b.sites(), "sites after the refused restores")
    a.restore(bytes(blob))
    a.step(7)
    b2 = _ctx(system, fils, sites)
    b2.step(12)
    assert_same(a.sites(), b2.sites(), "sites after a good restore")


def test_noise_key():
    """sc_set_noise_key before the first step gives the stream of a context
    created with that seed."""
    system, fils, sites = _workload("B", 0.02, seed=12)
    a = _ctx(dict(system, seed=5), fils, sites)
    a.set_noise_key(77)
    b = _ctx(dict(system, seed=77), fils, sites)
    a.step_graph(20)
    b.step_graph(20)
    assert_same(a.sites(), b.sites(), "sites")


def test_non_finite_positions_are_reported():
    """A NaN position fails the next step with SC_ERR_NAN (device status
    word), without faulting: binning clamps the cell and flags it."""
    import simcore_b200 as sc
    system, fils, sites = _workload("B", 0.02, seed=13)
    ctx = _ctx(system, fils, sites, "mixed")
    bad = sites.copy()
    bad[5, 0] = np.nan
    ctx.set_sites(bad)
    with pytest.raises(sc.ScError) as e:
        ctx.step(4)
        ctx.synchronize()
    assert e.value.code == 3


@pytest.mark.parametrize("graph", [False, True])
def test_unphysical_displacement_is_reported(graph):
    """A filament moved by 80 (set_sites) accumulates 2 x 80^2 > 10000 in its
    displacement tracker at the next full step, which the reference rejects
    as an "Unphysical result" (include/simcore/species.hpp:114-118): the step
    fails with SC_ERR_UNPHYSICAL, host-driven and inside a captured run."""
    import simcore_b200 as sc
    system, fils, sites = _workload("B", 0.02, seed=14)
    ctx = _ctx(system, fils, sites, "mixed")
    ctx.step(2)
    moved = ctx.sites()
    moved[:11, 0] += 80.0  # the first filament
    ctx.set_sites(moved)
    with pytest.raises(sc.ScError) as e:
        if graph:
            ctx.step_graph(20)
        else:
            ctx.step(6)
        ctx.synchronize()
    assert e.value.code == 7  # SC_ERR_UNPHYSICAL


def test_replica_list_overflow_is_reported():
    """Independent systems keep fixed pair segments (half again the initial
    list, plus 1,024).  Squeezing one small system's filaments into 0.3 of
    its box (shifts far below the unphysical bound) multiplies its density by
    eleven; the rebuild that follows outgrows the segment:
    SC_ERR_LIST_OVERFLOW."""
    import simcore_b200 as sc
    from simcore_b200 import workloads
    system, fils, sites, reps = workloads.make_replicas("D", n_replicas=3, fil_scale=0.02,
                                                        seed=15)
    ctx = _ctx_replicas(system, fils, sites, reps, "mixed")
    ctx.step(2)
    xyz = ctx.sites()
    n0 = reps[0]["n_filaments"] * 17  # sites of system 0 (16 bonds a filament)
    xyz[:n0, :2] *= 0.3
    assert 0.7 * np.abs(xyz[:n0, :2]).max() / 0.3 < 65.0
    ctx.set_sites(xyz)
    with pytest.raises(sc.ScError) as e:
        ctx.step(8)
        ctx.synchronize()
    assert e.value.code == 4  # SC_ERR_LIST_OVERFLOW


def test_invalid_inputs_are_rejected():
    """Inputs the library cannot take fail with an error status and a
    message, before any device work: no filaments, inconsistent site counts,
    bad parameters, filaments past the 511-bond limit, cell grids too large
    to count, negative step counts."""
    import simcore_b200 as sc
    system, fils, sites = _workload("A", 0.05, seed=1)
    with pytest.raises(sc.ScError):
        _ctx(system, [], np.zeros((0, 3)))
    with pytest.raises(sc.ScError, match="n_sites_total"):
        _ctx(system, fils, sites[:-1])
    bad = [dict(f) for f in fils]
    bad[0]["length"] = 0.0
    with pytest.raises(sc.ScError, match="bad parameters"):
        _ctx(system, bad, sites)
    long_fil = dict(fils[0], length=400.0, min_bond_length=0.5)
    n = sc.filament_n_bonds(long_fil) + 1
    assert n > 512
    with pytest.raises(sc.ScError, match="511 bonds"):
        _ctx(system, [long_fil], np.zeros((n, 3)))
    # Cell grids are bounded while their size is still a double: a radius of
    # 2.4e6 (2^22 cells a side, whose cube wraps a 64-bit count to 0) and an
    # infinite one are refused on the host.
    for radius in (2.4e6, float("inf")):
        with pytest.raises(sc.ScError, match="radius|cell grid"):
            _ctx(dict(system, system_radius=radius), fils, sites)
    ctx = _ctx(system, fils, sites)
    with pytest.raises(sc.ScError):
        ctx.step(-1)
    ctx.step(2)  # the context is still usable


def test_getters_leave_the_trajectory_alone():
    """Reading state (geometry, forces, pairs, cells, checkpoint) between
    steps changes nothing in the mixed path, whose bond orientations come
    from the fast integrator."""
    system, fils, sites = _workload("B", 0.03, seed=14)
    a = _ctx(system, fils, sites, "mixed")
    b = _ctx(system, fils, sites, "mixed")
    for n in (7, 30):
        a.step_graph(n)
        b.step_graph(n)
        a.bond_geometry()
        a.bond_forces()
        a.pairs()
        a.bond_cells()
        a.checkpoint()
    a.step_graph(21)
    b.step_graph(21)
    assert_same(a.sites(), b.sites(), "sites")


def test_reference_format_output(tmp_path):
    """Spec and posit files in the reference's format, at its cadence: every
    spec frame holds the sites of that step bit for bit; every posit frame the
    average position (reference summation order), its periodic image and the
    normalised average orientation."""
    import simcore_b200 as sc
    from ref_formats import read_posit, read_spec
    system, fils, sites = _workload("B", 0.01, seed=15)
    ctx = _ctx(system, fils, sites)
    run = str(tmp_path / "specrun")
    ctx.output_open(run, n_steps=60, n_posit=10, n_spec=20)
    expect_sites, expect_u = [], []
    for i in range(61):
        if i:
            ctx.step(1)
        ctx.output_write()
        if i % 20 == 0:
            expect_sites.append(ctx.sites())
        if i % 10 == 0:
            expect_u.append((ctx.sites(), ctx.bond_geometry()[2]))
    ctx.output_close()
    head, frames = read_spec(run + "_filament_filament.spec")
    assert head == (60, 20, system["delta"]) and len(frames) == 4
    ns = np.array([sc.filament_n_bonds(f) + 1 for f in fils])
    off = np.concatenate([[0], np.cumsum(ns)])
    for fr, xyz in zip(frames, expect_sites):
        assert len(fr) == len(fils)
        for k, rec in enumerate(fr):
            assert_same(rec["sites"], xyz[off[k]:off[k + 1]], "spec sites")
            assert rec["bending_stiffness"] == fils[k]["persistence_length"] and rec["poly"] == 0
    head, pframes = read_posit(run + "_filament_filament.posit")
    assert head == (60, 10, system["delta"]) and len(pframes) == 7
    R = system["system_radius"]
    for rec, (xyz, u) in zip(pframes, expect_u):
        for k in range(len(fils)):
            p = np.zeros(3)
            for s in xyz[off[k]:off[k + 1]]:
                p = p + s
            p = p / ns[k]
            assert_same(rec[k, 0:3], p, "posit average position")
            bu = u[off[k] - k:off[k + 1] - k - 1]
            a = np.zeros(3)
            for v in list(bu) + [bu[-1]]:
                a = a + v
            a = a / np.sqrt((a * a).sum())
            assert np.abs(rec[k, 6:9] - a).max() < 1e-14
            s_img = p / (2 * R)
            s_img -= np.where(s_img < 0, np.ceil(s_img - 0.5), np.floor(s_img + 0.5))
            assert np.abs(rec[k, 3:6] - s_img).max() < 1e-14
            assert rec[k, 9] == fils[k]["diameter"] and rec[k, 10] == fils[k]["length"]


def test_device_analyses_match_host():
    """On-device analyses of three independent 2D systems against the same
    quantities computed on the host from the sites and bond orientations:
    mean-square end-to-end distance and its standard error over samples,
    joint-angle histograms (exact counts), polar and nematic order."""
    import simcore_b200 as sc
    system, fils, sites, reps = _replica_batch(3, 0.03, seed=5)
    ctx = _ctx_replicas(system, fils, sites, reps)
    nb_bins = 50
    ns = np.array([sc.filament_n_bonds(f) + 1 for f in fils])
    off = np.concatenate([[0], np.cumsum(ns)])
    rep_of = np.repeat(np.arange(len(reps)), [r["n_filaments"] for r in reps])
    R = len(reps)
    m1, m2 = np.zeros(R), np.zeros(R)
    hist = np.zeros((R, ns.max() - 2, nb_bins), dtype=np.int64)
    for sample in range(5):
        ctx.step_graph(10)
        ctx.analysis_sample(nb_bins)
        xyz = ctx.sites()
        u = ctx.bond_geometry()[2]
        for f in range(len(fils)):
            p = xyz[off[f]:off[f + 1]]
            t = p[-1] - p[0]
            e = t[0] * t[0] + t[1] * t[1]
            m1[rep_of[f]] += e
            m2[rep_of[f]] += e * e
            bu = u[off[f] - f:off[f + 1] - f - 1]
            for j in range(len(bu) - 1):
                c = bu[j, 0] * bu[j + 1, 0] + bu[j, 1] * bu[j + 1, 1]
                b = min(max(int(np.floor((1 + c) * (nb_bins // 2))), 0), nb_bins - 1)
                hist[rep_of[f], j, b] += 1
    mse, err, n, h = ctx.analysis_results(nb_bins)
    assert n == 5
    num = np.array([r["n_filaments"] for r in reps], dtype=float)
    want = m1 / (5 * num)
    want_err = np.sqrt((m2 / (5 * num) - want * want) / (num * 5))
    assert np.allclose(mse, want, rtol=1e-12) and np.allclose(err, want_err, rtol=1e-9)
    assert (h == hist).all()
    polar, nem = ctx.global_order()
    u = ctx.bond_geometry()[2]
    for r in range(R):
        fs = np.where(rep_of == r)[0]
        pv = np.zeros(3)
        q = np.zeros((3, 3))
        for f in fs:
            bu = u[off[f] - f:off[f + 1] - f - 1][:, :2]
            pv[:2] += bu.mean(0)
            q[:2, :2] += (2 * np.einsum("bi,bj->ij", bu, bu) - len(bu) * np.eye(2)) / len(bu)
        assert np.allclose(polar[r], pv / len(fs), atol=1e-12)
        assert np.allclose(nem[r].reshape(3, 3), q / len(fs), atol=1e-12)
