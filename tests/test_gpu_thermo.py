"""GPU thermo: the pair virial, pressure records and potential energies.

The reference sums every pair's stress -dr x F into InteractionManager::
stress_ every step and turns it into the pressure tensor every n_thermo steps
(src/interaction_manager.cpp:500-517, 535-559).  The oracle does the same bit
for bit against the reference's own code (test_oracle.py).  The GPU sums the
virial in a fixed tree order instead of the serial one, so its pressures
agree with the oracle's to rounding -- within 1e-12 of the largest tensor
entry -- and are the same bits on every run and on both launch paths.  Per-
filament potential energies follow the reference's per-bond order and are
bit-identical in FP64.
"""
import struct

import numpy as np
import pytest

from checkers import Oracle
from test_gpu_parity import _ctx, _ctx_replicas, _replica_batch, _workload, assert_same

pytestmark = pytest.mark.gpu


def _close(a, b, rel, what):
    scale = np.abs(b).max()
    err = np.abs(np.asarray(a) - np.asarray(b)).max()
    assert err <= rel * scale, (what, err, scale)


@pytest.mark.parametrize("graph", [False, True])
def test_thermo_fp64_matches_oracle(graph):
    system, fils, sites = _workload("A", 1.0, seed=4)
    ctx = _ctx(system, fils, sites)
    o = Oracle(system, fils, sites)
    ctx.set_thermo(10)
    o.set_thermo(10)
    total = 0
    for n in (100, 101, 99):
        (ctx.step_graph if graph else ctx.step)(n)
        o.step(n)
        a, b = ctx.thermo_records(), o.thermo_records()
        assert np.array_equal(a[0], b[0])
        assert np.array_equal(a[3], b[3])
        _close(a[1], b[1], 1e-12, "pressure tensor")
        _close(a[2], b[2], 1e-12, "pressure")
        assert_same(ctx.potential_energy(), o.potential_energy(), "potential energy")
        assert_same(ctx.sites(), o.sites(), "sites")
        total += len(a[0])
    assert total == 30
    assert ctx.counters().n_rebuilds > 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_thermo_same_bits_on_both_paths_through_regrowth(precision):
    """Captured and host-driven runs give the same records, also when the
    captured run stops at an overflowing rebuild and resumes (buckling
    stiff filaments, five-fold pair growth)."""
    system, fils, sites = _workload("E", 0.1, seed=3)
    a = _ctx(system, fils, sites, precision)
    b = _ctx(system, fils, sites, precision)
    for c in (a, b):
        c.set_thermo(8)
    a.step_graph(400)
    b.step(400)
    assert a.counters().n_list_regrowths > 0
    ra, rb = a.thermo_records(), b.thermo_records()
    assert len(ra[0]) == 50
    for x, y in zip(ra, rb):
        assert_same(x, y, "records")
    assert_same(a.potential_energy(), b.potential_energy(), "potential energy")


def test_thermo_mixed_close_to_fp64():
    """The mixed path's virial from FP32 pair forces: the first record, taken
    on identical positions, within 1e-5 of the FP64 one."""
    system, fils, sites = _workload("B", 0.05, seed=8)
    a = _ctx(system, fils, sites, "fp64")
    b = _ctx(system, fils, sites, "mixed")
    for c in (a, b):
        c.set_thermo(1)
        c.step(1)
    ra, rb = a.thermo_records(), b.thermo_records()
    _close(rb[1], ra[1], 1e-5, "pressure tensor")
    _close(b.potential_energy(), a.potential_energy(), 1e-5, "potential energy")


def test_thermo_replicas_match_single_systems():
    from simcore_b200 import workloads
    system, fils, sites, reps = _replica_batch(4, 0.05, seed=5)
    batch = _ctx_replicas(system, fils, sites, reps)
    batch.set_thermo(4)
    batch.step_graph(40)
    st, P, p, V = batch.thermo_records()
    assert P.shape == (10, 4, 9)
    pote = batch.potential_energy()
    f0 = 0
    for r, part in enumerate(workloads.split_replicas(system, fils, sites, reps)):
        one = _ctx(*part)
        one.set_thermo(4)
        one.step_graph(40)
        s1, P1, p1, V1 = one.thermo_records()
        assert np.array_equal(s1, st)
        assert np.array_equal(V1, V[:, r])
        _close(P[:, r], P1, 1e-12, "pressure tensor")
        nf = len(part[1])
        assert_same(pote[f0:f0 + nf], one.potential_energy(), "potential energy")
        f0 += nf


def test_thermo_file(tmp_path):
    """The .thermo file: OutputManager::InitThermo's header (n_steps,
    n_thermo, delta, n_dim) and WriteThermo's records (unit cell, pressure
    tensor, pressure, volume)."""
    system, fils, sites = _workload("A", 1.0, seed=2)
    ctx = _ctx(system, fils, sites)
    ctx.set_thermo(5)
    run = str(tmp_path / "run")
    ctx.thermo_open(run, 50)
    ctx.step_graph(50)
    st, P, p, V = ctx.thermo_records()
    ctx.set_thermo(0)
    raw = open(run + ".thermo", "rb").read()
    n_steps, n_thermo, delta, n_dim = struct.unpack("<iidi", raw[:20])
    assert (n_steps, n_thermo, delta, n_dim) == (50, 5, system["delta"], 3)
    rec = np.frombuffer(raw[20:], dtype="<f8").reshape(-1, 20)
    assert rec.shape[0] == 10
    side = 2 * system["system_radius"]
    assert np.array_equal(rec[:, :9], np.tile([side, 0, 0, 0, side, 0, 0, 0, side], (10, 1)))
    assert np.array_equal(rec[:, 9:18], P)
    assert np.array_equal(rec[:, 18], p)
    assert np.array_equal(rec[:, 19], V)


def test_thermo_checkpoint_restore():
    """The pair records and running virial sums are part of a checkpoint:
    the restored run's records are the original's."""
    system, fils, sites = _workload("A", 1.0, seed=3)
    a = _ctx(system, fils, sites)
    a.set_thermo(6)
    a.step(15)
    blob = a.checkpoint()
    a.thermo_records()
    b = _ctx(system, fils, sites)
    b.set_thermo(6)
    b.restore(blob)
    a.step_graph(31)
    b.step_graph(31)
    ra, rb = a.thermo_records(), b.thermo_records()
    assert list(ra[0]) == [18, 24, 30, 36, 42]
    for x, y in zip(ra, rb):
        assert_same(x, y, "records")


def test_thermo_needs_enabling_for_potentials():
    import simcore_b200 as sc
    system, fils, sites = _workload("A", 1.0, seed=1)
    ctx = _ctx(system, fils, sites)
    with pytest.raises(sc.ScError):
        ctx.potential_energy()
