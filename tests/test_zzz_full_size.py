"""Workload B at its full size -- 20,000 filaments of 10 bonds in a periodic
cube of side 200, the headline configuration -- checked through properties
that do not depend on size:

* mixed-precision bond forces and torques within 1e-5 (max |d| / max) of
  the FP64 path's on the same state, on the state the benchmark starts from;
* a captured FP64 run through device-decided rebuilds gives the bits of the
  host-driven run;
* Newton's third law: a pair adds F to one bond and -F to the other, so the
  FP64 bond forces sum to zero up to rounding.

The file is named to be collected last, so that a run stopping at the first
failure has run every smaller test before it."""
import numpy as np
import pytest

from test_gpu_parity import _ctx, assert_same

pytestmark = pytest.mark.gpu


def _full_B(seed):
    from simcore_b200 import workloads
    return workloads.make("B", 1.0, seed=seed)


def test_full_size_B_mixed_force_error():
    system, fils, sites = _full_B(0)  # the benchmark's state (seed of rank 0)
    assert len(fils) == 20000
    c64 = _ctx(system, fils, sites, "fp64")
    c32 = _ctx(system, fils, sites, "mixed")
    c64.interact()
    c32.interact()
    f64, t64 = c64.bond_forces()
    f32, t32 = c32.bond_forces()
    assert c64.counters().n_pairs > 100000
    ef = np.abs(f32 - f64).max() / np.abs(f64).max()
    et = np.abs(t32 - t64).max() / np.abs(t64).max()
    assert ef <= 1e-5, ef
    assert et <= 1e-5, et
    # Newton's third law, in FP64: the total is rounding of the largest terms.
    assert np.abs(f64.sum(axis=0)).max() <= 1e-9 * np.abs(f64).sum()
    c64.close()
    c32.close()


def test_full_size_B_graph_matches_host():
    system, fils, sites = _full_B(1)
    a = _ctx(system, fils, sites, "fp64")
    b = _ctx(system, fils, sites, "fp64")
    a.step_graph(40)
    b.step(40)
    assert a.counters().n_rebuilds == b.counters().n_rebuilds > 1
    assert_same(a.sites(), b.sites(), "sites")
    assert_same(a.pairs(), b.pairs(), "pairs")
    a.close()
    b.close()
