"""Mixed precision against FP64, output by output, along trajectories.

Every output of the mixed path -- bond forces and torques, site forces,
tensions and the displacement of one step with shared noise -- stays within
1e-5 (max |mixed - fp64| / max |fp64|) of the FP64 path on the same state,
with the default settings (nearly parallel pairs side by side evaluated from
the FP64 sites), and in the nematic case with the near-parallel threshold
raised.  The states are snapshots of mixed-precision trajectories, where
close and nearly parallel contacts form: a dense isotropic suspension, a
nematic one of uneven lengths (nearly parallel pairs everywhere), a batch of
independent 2D systems, and a tethered network of buckling filaments.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = 1e-5


def _trajectory_errors(system, fils, sites, replicas=None, crosslinks=None, n_snap=4,
                       every=40, threshold=None):
    import simcore_b200 as sc
    from simcore_b200.accuracy import mixed_errors, max_errors
    ctx = sc.Context(system, fils, sites, precision="mixed", replicas=replicas)
    if crosslinks is not None:
        a, b, k, rest = crosslinks
        ctx.add_crosslinks(a, b, k_spring=k, rest_length=rest)
    errs = [mixed_errors(system, fils, sites, replicas, crosslinks,
                         near_parallel_threshold=threshold)]
    for _ in range(n_snap):
        ctx.step_graph(every)
        errs.append(mixed_errors(system, fils, ctx.sites(), replicas, crosslinks,
                                 near_parallel_threshold=threshold))
    ctx.close()
    return max_errors(errs), errs


def _check(errs):
    worst, _ = errs
    for name, e in worst.items():
        assert e <= BOUND, (name, e, worst)


def test_mixed_errors_isotropic_suspension():
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("B", 0.05, seed=21)
    _check(_trajectory_errors(system, fils, sites))


def test_mixed_errors_nematic_uneven_lengths():
    """Workload C's stiffness spread and nematic insertion with 20-bond
    filaments in a dense box (500 filaments, side 40: about 28,000 contacts).
    Nematic insertion starts every filament exactly parallel (both
    precisions take the parallel branch); the noise then turns them by small
    angles, which is where FP32 orientations cannot resolve closest points.
    Contacts a few degrees from parallel are everywhere here, so the FP64
    evaluation covers side-by-side pairs up to |u1 x u2|^2 = 1e-2 (about 6
    degrees; sc_set_near_parallel_threshold): every output then stays within
    1e-5 (the bond torque at 3.6e-6).  At the default 1e-5 the torque error of
    these states is 1.1e-5."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("C", 0.01, seed=22, n_seg=20, side=40.0)
    _check(_trajectory_errors(system, fils, sites, every=60, threshold=1e-2))


def test_mixed_errors_replica_batch():
    from simcore_b200 import workloads
    system, fils, sites, reps = workloads.make_replicas("D", n_replicas=4, fil_scale=0.2,
                                                        seed=23)
    _check(_trajectory_errors(system, fils, sites, replicas=reps))


def test_mixed_errors_tethered_network():
    """Workload E's density, stiffness and tethers with 10-bond filaments, so
    that filaments are shorter than the small box (longer ones would overlap
    their own periodic images)."""
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("E", 0.02, seed=24, n_seg=10)
    xl = workloads.crosslinks("E", sites, fils, 2 * system["system_radius"], scale=0.02,
                              seed=24)
    _check(_trajectory_errors(system, fils, sites, crosslinks=xl, every=30))


def test_near_parallel_pairs_off_is_the_fp32_evaluation():
    """The default mixed path evaluates a pair at 1.7e-4 rad from the FP64
    sites (within the bound of the FP64 torques); with that evaluation
    switched off the pair is evaluated in FP32, from orientations that
    cannot resolve its closest points, and the torques change."""
    import simcore_b200 as sc
    angle = 1.7e-4
    j = np.arange(11.0)
    sites = np.zeros((22, 3))
    sites[:11, 0] = j - 5.0
    sites[11:, 0] = -4.7 + j * np.cos(angle)
    sites[11:, 2] = 1.05 + j * np.sin(angle)
    system = dict(n_dim=3, system_radius=20.0, delta=1e-4, seed=1, stoch_flag=0)
    fils = [dict(length=10.0, persistence_length=100.0, diameter=1.0, min_bond_length=0.666,
                 friction_ratio=2.0)] * 2
    out = {}
    for mode in ("fp64", "mixed", "mixed_off"):
        c = sc.Context(system, fils, sites, precision="fp64" if mode == "fp64" else "mixed")
        if mode == "mixed_off":
            c.set_exact_near_parallel(False)
        c.interact()
        out[mode] = c.bond_forces()
        c.close()
    t64 = out["fp64"][1]
    scale = max(np.abs(t64).max(), np.abs(out["fp64"][0]).max())
    assert np.abs(out["mixed"][1] - t64).max() <= BOUND * scale
    assert not np.array_equal(out["mixed_off"][1], out["mixed"][1])
