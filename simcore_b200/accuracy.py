"""Accuracy of the mixed-precision path against the FP64 path, output by output.

The FP64 path is bit-identical to the reference's CPU code.  The mixed path
evaluates pair geometry and WCA forces in FP32 (nearly parallel pairs side by
side in FP64) and runs the fast integrator: FP64 bending, tension solve and
positions, the midstep noise drawn and projected in FP32.  mixed_errors() loads one state into
a fresh context of each precision -- fresh pair lists and no stale pair
forces, so both evaluate exactly the same pairs -- and compares, as
max |mixed - fp64| / max |fp64| over all entries:

  bond_force, bond_torque  Bond::force_ / torque_ after Interact;
  site_force               the total force on every site in the integrator
                           step that follows (interaction, bending, noise,
                           tension forces);
  tension                  the tension of every bond in that step;
  displacement             r_after - r_before of every site over that step
                           (a midstep: both contexts draw the same noise).

Called on a trajectory's snapshots it gives the error along the trajectory
("shadow" FP64 evaluations of the mixed run's own positions).
"""
import numpy as np

from . import Context

OUTPUTS = ("bond_force", "bond_torque", "site_force", "tension", "displacement")


def _rel(a, b):
    scale = float(np.abs(b).max())
    return float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a).max())


def mixed_errors(system, filaments, sites, replicas=None, crosslinks=None, device=0,
                 near_parallel_threshold=None):
    """Max relative error of every output of the mixed path against FP64 on
    the state `sites` (see the module docstring).  crosslinks: optional
    (site_a, site_b, k_spring, rest_length) of static tethers.
    near_parallel_threshold: the mixed context's threshold on |u1 x u2|^2
    (sc_set_near_parallel_threshold), when not the default."""
    res = {}
    for prec in ("fp64", "mixed"):
        ctx = Context(system, filaments, sites, precision=prec, device=device,
                      replicas=replicas)
        try:
            if prec == "mixed" and near_parallel_threshold is not None:
                ctx.set_near_parallel_threshold(near_parallel_threshold)
            if crosslinks is not None:
                a, b, k, rest = crosslinks
                ctx.add_crosslinks(a, b, k_spring=k, rest_length=rest)
            ctx.set_capture(True)
            before = ctx.sites()
            ctx.interact()
            f, t = ctx.bond_forces()
            ctx.update_positions()
            res[prec] = dict(bond_force=f, bond_torque=t, site_force=ctx.site_forces(),
                             tension=ctx.tensions(), displacement=ctx.sites() - before)
        finally:
            ctx.close()
    return {k: _rel(res["mixed"][k], res["fp64"][k]) for k in OUTPUTS}


def max_errors(list_of_errors):
    """Entry-wise maximum of several mixed_errors() results."""
    return {k: max(e[k] for e in list_of_errors) for k in OUTPUTS}
