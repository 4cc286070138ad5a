"""With sc_set_fused_pairs the fast mixed step evaluates each bond's pairs
inside the integrator instead of launching the pair stage.  It must give the
bits of the split
interface, sc_interact (the separate pair stage, per-bond slots) followed by
sc_update_positions (the integrator summing those slots), over runs with
rebuilds, in both integrator kernels, with replicas and with tethers.  After
a fused step the bond-force getter returns the step's pair evaluation, as
after the pair stage."""
import numpy as np
import pytest

from test_gpu_parity import _ctx, _ctx_replicas, _replica_batch, _workload, _workload_E, assert_same

pytestmark = pytest.mark.gpu


def _split(ctx, n):
    for _ in range(n):
        ctx.interact()
        ctx.update_positions()


def _pair(case):
    """Two contexts of one mixed-precision workload, the first fused.  The
    fusion evaluates every pair in FP32, so both contexts run with the FP64
    evaluation of nearly parallel pairs (on by default) switched off."""
    a, b = _contexts(case)
    for c in (a, b):
        c.set_exact_near_parallel(False)
    a.set_fused_pairs(True)
    return a, b


def _contexts(case):
    if case == "B":  # 11-site filaments: the block integrator
        system, fils, sites = _workload("B", 0.05, seed=6)
        return _ctx(system, fils, sites, "mixed"), _ctx(system, fils, sites, "mixed")
    if case == "C":  # 6 to 201 sites: warp and block integrators together
        system, fils, sites = _workload("C", 0.002, seed=3, side=150.0)
        out = []
        for _ in range(2):
            c = _ctx(system, fils, sites, "mixed")
            c.set_integrator_layout(32, 256)
            out.append(c)
        return tuple(out)
    if case == "D":  # several 2D systems in one context
        system, fils, sites, reps = _replica_batch(4, 0.03, seed=2)
        return (_ctx_replicas(system, fils, sites, reps, "mixed"),
                _ctx_replicas(system, fils, sites, reps, "mixed"))
    system, fils, sites, (a, b, k, rest) = _workload_E(0.01, seed=4)  # tethers
    out = []
    for _ in range(2):
        c = _ctx(system, fils, sites, "mixed")
        c.add_crosslinks(a, b, k_spring=k, rest_length=rest)
        out.append(c)
    return tuple(out)


def _same_state(a, b):
    assert_same(a.sites(), b.sites(), "sites")
    assert_same(a.prev_sites(), b.prev_sites(), "prev sites")
    assert_same(a.pairs(), b.pairs(), "pair list")
    fa, ta = a.bond_forces()
    fb, tb = b.bond_forces()
    assert_same(fa, fb, "bond forces")
    assert_same(ta, tb, "bond torques")
    assert a.counters().n_rebuilds == b.counters().n_rebuilds


@pytest.mark.parametrize("case", ["B", "C", "D", "E"])
def test_fused_step_matches_split_interface(case):
    a, b = _pair(case)
    for n in (1, 2, 17, 40):
        a.step(n)
        _split(b, n)
        _same_state(a, b)
    if case in ("B", "C"):
        assert a.counters().n_rebuilds > 1  # the run crossed rebuilds
    # The slots the getter wrote are the ones the pair stage leaves, so the
    # state after it is unchanged: the runs still agree.
    a.step(5)
    _split(b, 5)
    _same_state(a, b)


@pytest.mark.parametrize("case", ["B", "C"])
def test_fused_graph_matches_split_interface(case):
    a, b = _pair(case)
    for n in (40, 41):
        a.step_graph(n)
        _split(b, n)
        _same_state(a, b)


def test_fused_launches_no_pair_stage():
    """A captured run of the fused step launches two kernels fewer per BD
    step than the same run with the pair stage; thermo, which needs the
    pair stage's records, turns the fusion off."""
    a, b = _pair("B")
    l0a, l0b = a.counters().kernel_launches, b.counters().kernel_launches
    a.step_graph(40)
    b.step_graph(40)
    la, lb = a.counters(), b.counters()
    assert_same(a.sites(), b.sites(), "sites")
    assert la.n_rebuilds == lb.n_rebuilds
    assert (lb.kernel_launches - l0b) - (la.kernel_launches - l0a) == 20 * 2
    a.set_thermo(10 ** 6)  # records every 10^6 steps: none in range
    b.set_thermo(10 ** 6)
    l0a, l0b = a.counters().kernel_launches, b.counters().kernel_launches
    a.step_graph(40)
    b.step_graph(40)
    assert_same(a.sites(), b.sites(), "sites")
    assert (b.counters().kernel_launches - l0b) == (a.counters().kernel_launches - l0a)


def test_bond_forces_after_set_sites_are_the_last_evaluation():
    """sc_set_sites between a fused step and the getter leaves the step's
    pair evaluation readable (the split interface's slots are not touched by
    it either)."""
    a, b = _pair("B")
    a.step(3)
    _split(b, 3)
    xyz = a.sites()
    moved = xyz + 0.01
    a.set_sites(moved)
    b.set_sites(moved)
    fa, ta = a.bond_forces()
    fb, tb = b.bond_forces()
    assert_same(fa, fb, "bond forces")
    assert_same(ta, tb, "bond torques")
    assert np.abs(fa).max() > 0
    a.step(4)
    _split(b, 4)
    _same_state(a, b)
