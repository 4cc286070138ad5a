"""sc_pair_forces_noalloc: pair forces for callers that cannot allocate.

An application whose device memory belongs to its own pool or caching
allocator must not have it grown behind its back, and one that runs under a
device-memory budget fixed at start-up cannot call cudaMalloc at all; the
no-allocation entry point serves both by working in a fixed scratch array
inside the library.  This test calls it through the C ABI on buffers the
test owns and checks its bond forces and torques against those of the
regular entry points (sc_interact on a context just loaded with the same
sites) -- FP64, so exactly equal -- on two calls in a row, the second
finding the first call's data still in the scratch.

The file is named to be collected last, so that a run stopping at the first
failure has already run every other test.  It passes alone in a fresh
process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_forces(system, fils, sites):
    import simcore_b200 as sc
    ctx = sc.Context(system, fils, sites, precision="fp64")
    ctx.interact()
    f, t = ctx.bond_forces()
    ctx.close()
    return f, t


def _site_offsets(fils):
    import simcore_b200 as sc
    n_bonds = [sc.filament_n_bonds(f) for f in fils]
    offsets = np.zeros(len(fils) + 1, dtype=np.int32)
    offsets[1:] = np.cumsum(np.asarray(n_bonds) + 1)
    return offsets


def _call_noalloc(system, fils, sites, offsets=None, expect=0):
    """Calls the entry point on test-owned device buffers; returns the bond
    forces and torques when it is expected to succeed (expect = 0)."""
    import torch

    import simcore_b200 as sc
    n_bonds = [sc.filament_n_bonds(f) for f in fils]
    if offsets is None:
        offsets = _site_offsets(fils)
    nb = int(sum(n_bonds))
    d_off = torch.from_numpy(offsets).cuda()
    d_xyz = torch.from_numpy(np.ascontiguousarray(sites, dtype=np.float64)).cuda()
    d_f = torch.full((nb, 3), float("nan"), dtype=torch.float64, device="cuda")
    d_t = torch.full((nb, 3), float("nan"), dtype=torch.float64, device="cuda")
    desc = sc.SystemDesc(n_dim=system["n_dim"], system_radius=system["system_radius"],
                         delta=system["delta"], wca_eps=1.0, wca_sig=1.0, f_cutoff=2000.0,
                         stoch_flag=1, interaction_flag=1, like_like_interactions=1,
                         seed=system.get("seed", 0), precision=0, device=0)
    species = sc.FilamentParams(**fils[0])
    stream = torch.cuda.current_stream().cuda_stream
    rc = sc.lib.sc_pair_forces_noalloc(
        ctypes.byref(desc), ctypes.byref(species), ctypes.c_int(len(fils)),
        ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_xyz.data_ptr()),
        ctypes.c_void_p(d_f.data_ptr()), ctypes.c_void_p(d_t.data_ptr()),
        ctypes.c_void_p(stream))
    assert rc == expect, sc.STATUS_NAMES.get(rc, rc)
    return d_f.cpu().numpy(), d_t.cpu().numpy()


def test_noalloc_matches_regular_entry_points_twice():
    from simcore_b200 import workloads
    cases = [workloads.make("A", 0.5, seed=11), workloads.make("B", 0.02, seed=12)]
    for system, fils, sites in cases:
        f_ref, t_ref = _reference_forces(system, fils, sites)
        assert np.abs(f_ref).max() > 0  # the configuration has interacting pairs
        for _ in range(2):
            f, t = _call_noalloc(system, fils, sites)
            assert np.array_equal(f, f_ref)
            assert np.array_equal(t, t_ref)


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    import simcore_b200 as sc
    too_many = 8192 + 1  # filaments; SC_NOALLOC_MAX_BONDS
    desc = sc.SystemDesc(n_dim=3, system_radius=50.0, delta=1e-4, wca_eps=1.0, wca_sig=1.0,
                         f_cutoff=2000.0, stoch_flag=1, interaction_flag=1,
                         like_like_interactions=1, seed=0, precision=0, device=0)
    species = sc.FilamentParams(length=10.0, persistence_length=100.0, diameter=1.0,
                                min_bond_length=0.666, friction_ratio=2.0)
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    o = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = sc.lib.sc_pair_forces_noalloc(
        ctypes.byref(desc), ctypes.byref(species), ctypes.c_int(too_many),
        ctypes.c_void_p(o.data_ptr()), ctypes.c_void_p(d.data_ptr()),
        ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(0))
    assert rc == 1  # SC_ERR_INVALID_ARG


def test_noalloc_rejects_bad_site_offsets():
    """The site offsets are device data that the host does not read: the
    unpack kernel checks them (rising from 0 by at least 2 sites a filament)
    and the call returns SC_ERR_INVALID_ARG, writing nothing outside its
    scratch.  A correct call afterwards gives the regular forces."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("A", 0.1, seed=13)
    good = _site_offsets(fils)
    swapped = good.copy()
    swapped[1], swapped[2] = good[2], good[1]  # filament 1 runs backwards
    short = good.copy()
    short[1] = 1                                # a filament of one site
    for bad in (swapped, short):
        assert bad[0] == 0 and bad[-1] == good[-1]  # only the device check can see it
        _call_noalloc(system, fils, sites, offsets=bad, expect=1)  # SC_ERR_INVALID_ARG
    f_ref, t_ref = _reference_forces(system, fils, sites)
    f, t = _call_noalloc(system, fils, sites)
    assert np.array_equal(f, f_ref)
    assert np.array_equal(t, t_ref)


def test_noalloc_rejects_cell_grids_beyond_the_limit():
    """The cell count is bounded on the host while it is still a double: a
    large finite radius (2^22 cells a side would wrap a 64-bit cell count to
    0) and an infinite one are refused before any launch, and a correct call
    afterwards still gives the regular forces."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("A", 0.1, seed=14)
    for radius in (2.4e6, 1e300, float("inf"), 60.0):
        # 60: 104 cells a side in 3D, over the 50 the scratch holds
        big = dict(system, system_radius=radius)
        _call_noalloc(big, fils, sites, expect=1)  # SC_ERR_INVALID_ARG
    f_ref, t_ref = _reference_forces(system, fils, sites)
    f, t = _call_noalloc(system, fils, sites)
    assert np.array_equal(f, f_ref)
    assert np.array_equal(t, t_ref)
