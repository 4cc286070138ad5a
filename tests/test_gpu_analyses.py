"""On-device analyses against the reference's own analysis code.

The checker runs the reference's FilamentSpecies::RunMse2eAnalysis /
RunThetaAnalysis / FinalizeMse2eAnalysis and its diffusion analysis
(SpherocylinderSpecies' time-origin averaged MSD and orientation
correlation, on the filaments' average positions and orientations) on the
reference's own Filament objects (oracle/_ref).  The GPU runs the same
simulation in FP64 (bit-identical states), so per-filament values are
identical and the per-system sums agree to rounding (another summation
order); histogram counts are equal.

The reference's joint-angle histogram reads the cosines its integrator took
at the start of the last step (Filament::GetThetas), so it sees the state one
step behind its end-to-end distances; the GPU's histogram of a state is the
reference's of the next step.
"""
import numpy as np
import pytest

from checkers import Reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not Reference.available(),
                                 reason="reference build not present")]


def _case(n_dim):
    import simcore_b200 as sc
    nb = np.full(30, 12, dtype=np.int32)
    R = 14.0 if n_dim == 3 else 30.0
    sites = sc.insert_filaments(n_dim, R, 5, nb, nb.astype(float), np.full(30, 20.0))
    system = dict(n_dim=n_dim, system_radius=R, delta=2e-4, seed=5)
    fils = [dict(length=12.0, persistence_length=20.0, diameter=1.0, min_bond_length=0.666,
                 friction_ratio=2.0)] * 30
    return system, fils, sites


@pytest.mark.parametrize("n_dim", [3, 2])
def test_end_to_end_and_angle_histograms_match_reference(n_dim):
    import simcore_b200 as sc
    system, fils, sites = _case(n_dim)
    ctx = sc.Context(system, fils, sites, precision="fp64")
    ref = Reference(system, fils, sites)
    n_bins = 40
    for steps in (7, 10, 10):
        ctx.step(steps)
        ref.step(steps)
        ctx.analysis_sample(n_bins)
        ref.analysis_sample(n_bins)
    m, e, ns, _ = ctx.analysis_results(n_bins)
    rm, re_, rns, _ = ref.analysis_results()
    assert ns == rns == 3
    assert abs(m[0] - rm) <= 1e-12 * rm
    assert abs(e[0] - re_) <= 1e-9 * re_
    ctx.close()
    ref.close()
    # The histogram of one state: the GPU after k steps, the reference after
    # k + 1 (its cosines of the state the (k+1)-th step started from).
    ctx = sc.Context(system, fils, sites, precision="fp64")
    ref = Reference(system, fils, sites)
    ctx.step(9)
    ref.step(10)
    ctx.analysis_sample(n_bins)
    ref.analysis_sample(n_bins)
    _, _, _, hist = ctx.analysis_results(n_bins)
    _, _, _, rhist = ref.analysis_results()
    assert rhist.shape == hist[0].shape
    assert np.array_equal(hist[0], rhist)
    assert rhist.sum() == 30 * 11
    ctx.close()
    ref.close()


@pytest.mark.parametrize("n_dim", [3, 2])
def test_com_diffusion_matches_reference(n_dim):
    """Time-origin averaged centre-of-mass MSD and orientation correlation,
    two windows of 4 samples, 6 steps apart."""
    import simcore_b200 as sc
    system, fils, sites = _case(n_dim)
    ctx = sc.Context(system, fils, sites, precision="fp64")
    ref = Reference(system, fils, sites)
    ctx.step(4)
    ref.step(4)
    ctx.diffusion_init(4)
    ref.diffusion_init(4)
    for _ in range(8):
        ctx.step(6)
        ref.step(6)
        ctx.diffusion_sample()
        ref.diffusion_sample()
    got = ctx.diffusion_results()
    want = ref.diffusion_results()
    # The weights are inverse variances over the filaments, <x^2> - <x>^2: for
    # the orientation correlation (x = u . u0 close to 1) that difference
    # cancels most digits, so another summation order moves its relative
    # value by ~1e-8.
    for g, w, name, rtol in zip(got, want, ("msd", "msd_err", "vcf", "vcf_err"),
                                (1e-9, 1e-9, 1e-6, 1e-6)):
        assert np.all(np.isfinite(w)), name
        assert np.allclose(g, w, rtol=rtol, atol=0), (name, g, w)
    assert np.all(np.diff(want[0]) > 0)  # the MSD grows through a window
    ctx.close()
    ref.close()
