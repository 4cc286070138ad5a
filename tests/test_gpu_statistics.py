"""Long-run statistics of the mixed-precision path.

The FP64 path is bit-identical to the reference, so its statistics are the
reference's.  The mixed path's trajectories diverge from it (FP32 pair forces,
contracted FP64 integrator); what must agree is the statistics.  Over 2,000
steps of 2,000 filaments (workload B's density and stiffness), these are
compared:
  * the mean-square end-to-end distance,
  * the centre-of-mass mean-square displacement,
  * the mean cosine between consecutive bonds.
The mixed run uses an independent noise stream (another seed), so the
comparison is statistical: the means agree within 3 standard errors of the
difference, with filaments as independent samples.  With the same noise
stream the two precisions stay within a tenth of a standard error.  The bond
cosine is checked against the worm-like-chain value coth(lp/l) - l/lp, which
the reference's insertion draws from (src/filament.cpp:350-383), to 1e-3: the
reference's dynamics settles about 3e-4 above it at dt = 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _observables(xyz, n_sites, xyz0):
    off = np.concatenate([[0], np.cumsum(n_sites)])
    r2, msd, cos = [], [], []
    for f in range(len(n_sites)):
        p = xyz[off[f]:off[f + 1]]
        p0 = xyz0[off[f]:off[f + 1]]
        r2.append(((p[-1] - p[0]) ** 2).sum())
        msd.append(((p.mean(0) - p0.mean(0)) ** 2).sum())
        u = np.diff(p, axis=0)
        u /= np.linalg.norm(u, axis=1)[:, None]
        cos.append((u[1:] * u[:-1]).sum(1).mean())
    return np.array(r2), np.array(msd), np.array(cos)


def _agree(a, b, what):
    se = np.sqrt(a.var() / len(a) + b.var() / len(b))
    assert abs(a.mean() - b.mean()) <= 3 * se, (what, a.mean(), b.mean(), se)


def test_mixed_statistics_match_fp64_over_long_runs():
    import simcore_b200 as sc
    from simcore_b200 import workloads
    system, fils, sites = workloads.make("B", 0.1, seed=11)
    n_sites = np.array([sc.filament_n_bonds(f) + 1 for f in fils])
    obs = {}
    for prec, seed in (("fp64", 11), ("mixed", 12), ("mixed_same", 11)):
        ctx = sc.Context(dict(system, seed=seed), fils, sites,
                         precision="fp64" if prec == "fp64" else "mixed")
        ctx.step_graph(2000)
        obs[prec] = _observables(ctx.sites(), n_sites, sites)
        ctx.close()
    for i, what in enumerate(("R_ee^2", "COM MSD", "bond cosine")):
        _agree(obs["mixed"][i], obs["fp64"][i], what)
        a, b = obs["mixed_same"][i], obs["fp64"][i]
        assert abs(a.mean() - b.mean()) <= 0.1 * b.std() / np.sqrt(len(b)), what
    k = fils[0]["persistence_length"] / 1.0
    wlc = 1.0 / np.tanh(k) - 1.0 / k
    for prec in ("fp64", "mixed"):
        assert abs(obs[prec][2].mean() - wlc) <= 1e-3, (prec, obs[prec][2].mean(), wlc)
    # The filaments diffused: the COM moved by far more than rounding.
    assert obs["fp64"][1].mean() > 1e-2
