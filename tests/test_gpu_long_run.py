"""Long-run statistics of the filament step against polymer theory.

Two runs of 200 filaments of 10 bonds (bond length 1, diameter 1, friction
ratio 2, WCA between filaments, noise on, dt 1e-4) in a dilute periodic box,
for each precision:

* Relaxation to the worm-like chain.  The filaments start straight (inserted
  with persistence length 1e6) but move with persistence length 5, so the
  end-to-end distance must relax from L^2 = 100 to the discrete chain's
  equilibrium.  With only bending energy kappa cos(theta) per joint
  (kappa = lp / l), the joint angles are independent with mean cosine
  c = coth(kappa) - 1/kappa, and
      <R^2> = l^2 [n (1 + c) / (1 - c) - 2 c (1 - c^n) / (1 - c)^2]
  (n bonds), 54.3 here.  (The reference's own analysis quotes the
  continuous chain, 2 L lp - 2 lp^2 (1 - exp(-L / lp)) = 56.8,
  src/filament_species.cpp:382; the model is the discrete chain.)  After
  2e5 steps (10 time units) the
  time average over the next 4e5 steps must match within three standard
  errors (filaments are the independent samples) plus 1%; the two halves of
  the window must agree (the run has relaxed).
* Centre-of-mass diffusion.  Stiff filaments (lp 100, as in the dense
  suspension workload) diffuse as rods with the reference's Doi-Edwards
  friction per site (src/filament.cpp:331-333): g_perp = 4 L / (3 N
  log(L/d)), g_par = g_perp / 2, so D = kT (1/g_par + 2/g_perp) / (3 N) =
  log(L/d) / L.  The MSD slope over lags up to one time unit (all time
  origins) must match 6 D within three standard errors plus 5%.  (At lp
  1000 and dt 1e-4 the reference's own integrator drives each filament
  along its axis -- its compiled code shows a lag-one correlation of 0.4
  between successive axial steps, which vanishes at dt 2.5e-5 -- so the
  rod limit is tested at lp 100.)

Time counts as the reference does: one i_step is dt/2 (a midstep or a full
step), sc_step_graph runs them in captured batches.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_FIL, N_SEG = 200, 10
DT = 1e-4


def _system(lp_insert, seed, side=60.0):
    import simcore_b200 as sc
    nb = np.full(N_FIL, N_SEG, dtype=np.int32)
    sites = sc.insert_filaments(3, side / 2, seed, nb, nb.astype(float),
                                np.full(N_FIL, lp_insert))
    system = dict(n_dim=3, system_radius=side / 2, delta=DT, seed=seed)
    return system, sites


def _fils(lp):
    return [dict(length=float(N_SEG), persistence_length=lp, diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * N_FIL


def _run(precision, system, sites, lp, n_equil, n_samples, every):
    import simcore_b200 as sc
    ctx = sc.Context(system, _fils(lp), sites, precision=precision)
    try:
        if n_equil:
            ctx.step_graph(n_equil)
        out = []
        for _ in range(n_samples):
            ctx.step_graph(every)
            out.append(ctx.sites().reshape(N_FIL, N_SEG + 1, 3))
        return np.array(out)  # samples x filaments x sites x 3
    finally:
        ctx.close()


def _wlc_discrete(lp, n, l=1.0):
    k = lp / l
    c = 1.0 / np.tanh(k) - 1.0 / k
    return l * l * (n * (1 + c) / (1 - c) - 2 * c * (1 - c ** n) / (1 - c) ** 2)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_end_to_end_distance_relaxes_to_the_worm_like_chain(precision):
    lp = 5.0
    system, sites = _system(1e6, seed=31)
    traj = _run(precision, system, sites, lp, n_equil=200000, n_samples=200, every=2000)
    r2 = ((traj[:, :, -1] - traj[:, :, 0]) ** 2).sum(-1)  # samples x filaments
    per_fil = r2.mean(0)
    mean, se = per_fil.mean(), per_fil.std(ddof=1) / np.sqrt(N_FIL)
    theory = _wlc_discrete(lp, N_SEG)
    assert abs(mean - theory) <= 3 * se + 0.01 * theory, (mean, se, theory)
    first, second = r2[:100].mean(0), r2[100:].mean(0)
    d = second - first
    assert abs(d.mean()) <= 3 * d.std(ddof=1) / np.sqrt(N_FIL) + 0.01 * theory, (
        first.mean(), second.mean())
    # The start was straight: the relaxation is far beyond the error bar.
    assert 100.0 - mean > 20 * se


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_centre_of_mass_diffusion_matches_doi_edwards(precision):
    lp = 100.0
    system, sites = _system(lp, seed=32)
    every = 1000  # i_steps: 0.05 time units
    traj = _run(precision, system, sites, lp, n_equil=0, n_samples=100, every=every)
    # Centres of mass, unwrapped: a filament's sites may be moved by a box
    # vector as one, so consecutive samples (0.26 sigma rms apart, box 60)
    # are joined by their minimum image.
    com = traj.mean(2)  # samples x filaments x 3
    side = 2 * system["system_radius"]
    step = np.diff(com, axis=0)
    step -= side * np.round(step / side)
    com = np.concatenate([com[:1], com[:1] + np.cumsum(step, axis=0)])
    dt_sample = every * DT / 2
    lags = np.arange(2, 21)  # 0.1 .. 1 time unit
    msd = np.array([((com[k:] - com[:-k]) ** 2).sum(-1).mean(0) for k in lags])  # lags x fil
    t = lags * dt_sample
    slope_per_fil = (msd * t[:, None]).sum(0) / (t * t).sum()  # fit through the origin
    slope, se = slope_per_fil.mean(), slope_per_fil.std(ddof=1) / np.sqrt(N_FIL)
    D = np.log(N_SEG / 1.0) / N_SEG
    assert abs(slope - 6 * D) <= 3 * se + 0.05 * 6 * D, (slope, se, 6 * D)
