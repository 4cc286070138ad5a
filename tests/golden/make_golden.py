"""Generates the golden fixtures of tests/golden/ from the reference's own
code (oracle/_ref/libscref.so, built from the reference sources by
oracle/ref/Makefile).  Run where the reference tree is present:

    python tests/golden/make_golden.py

Each fixture holds a seeded initial configuration (random insertion with
overlap rejection) and the reference's state after a fixed number of steps;
the thermo_* fixtures hold its pressure records and potential energies, the
format_* ones a spec and a posit frame as its own writers write them, the
tether_* ones a run with doubly-bound crosslinks of its own Crosslink and
Anchor code.
tests/test_oracle.py requires the C oracle to reproduce every array bit for
bit; the GPU tests require the CUDA path to match the oracle the same way.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from checkers import Reference  # noqa: E402

import simcore_b200 as sc  # noqa: E402

CASES = {
    # 3D, stiff filaments (workload A's physics) in a small dense box
    "ref3d_stiff": dict(n_dim=3, R=15.0, n_fil=20, n_seg=20, lp=500.0, delta=1e-4, seed=21,
                        steps=61),
    # 3D, flexible filaments: frequent renormalisations
    "ref3d_flexible": dict(n_dim=3, R=12.0, n_fil=30, n_seg=10, lp=5.0, delta=1e-3, seed=22,
                           steps=41),
    # 2D
    "ref2d": dict(n_dim=2, R=25.0, n_fil=40, n_seg=16, lp=200.0, delta=1e-4, seed=23,
                  steps=61),
}


def make_case(name, c):
    nb = np.full(c["n_fil"], c["n_seg"], dtype=np.int32)
    sites = sc.insert_filaments(c["n_dim"], c["R"], c["seed"], nb, nb.astype(float),
                                np.full(c["n_fil"], c["lp"]))
    system = dict(n_dim=c["n_dim"], system_radius=c["R"], delta=c["delta"], wca_eps=1.0,
                  wca_sig=1.0, f_cutoff=2000.0, stoch_flag=1, interaction_flag=1,
                  like_like_interactions=1, seed=c["seed"])
    fils = [dict(length=float(c["n_seg"]), persistence_length=c["lp"], diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * c["n_fil"]
    ref = Reference(system, fils, sites, n_threads=2)
    ref.step(c["steps"])
    f, t = ref.bond_forces()
    sw, nn = ref.filament_state()
    out = dict(
        system=np.array([c["n_dim"], c["R"], c["delta"], c["seed"], c["lp"], c["n_seg"],
                         c["n_fil"], c["steps"]], dtype=np.float64),
        sites0=sites, sites=ref.sites(), prev_sites=ref.prev_sites(),
        random_forces=ref.random_forces(), site_forces=ref.site_forces(), bond_force=f,
        bond_torque=t, tensions=ref.tensions(), pairs=ref.pairs(), dr_tot=ref.dr_tot(),
        normalize_switch=sw, n_normalize=nn, bond_cells=ref.bond_cells(),
        n_rebuilds=np.array([ref.n_rebuilds]))
    ref.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


# Pressure records (InteractionManager::CalculatePressure every n_thermo
# steps) and per-filament potential energies, from runs with rebuilds.
THERMO_CASES = {
    "thermo_3d": dict(n_dim=3, R=14.0, n_fil=25, n_seg=12, lp=50.0, delta=2e-4, seed=7,
                      insert_seed=102, steps=90, n_thermo=6),
    "thermo_2d": dict(n_dim=2, R=22.0, n_fil=30, n_seg=14, lp=50.0, delta=2e-4, seed=7,
                      insert_seed=101, steps=90, n_thermo=6),
}


def make_thermo_case(name, c):
    nb = np.full(c["n_fil"], c["n_seg"], dtype=np.int32)
    sites = sc.insert_filaments(c["n_dim"], c["R"], c["insert_seed"], nb, nb.astype(float),
                                np.full(c["n_fil"], c["lp"]))
    system = dict(n_dim=c["n_dim"], system_radius=c["R"], delta=c["delta"], seed=c["seed"])
    fils = [dict(length=float(c["n_seg"]), persistence_length=c["lp"], diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * c["n_fil"]
    ref = Reference(system, fils, sites, n_threads=2)
    ref.set_thermo(c["n_thermo"])
    ref.step(c["steps"])
    st, P, p, V = ref.thermo_records()
    out = dict(
        system=np.array([c["n_dim"], c["R"], c["delta"], c["seed"], c["lp"], c["n_seg"],
                         c["n_fil"], c["steps"]], dtype=np.float64),
        n_thermo=np.array([c["n_thermo"]]), sites0=sites, sites=ref.sites(),
        thermo_step=st, thermo_tensor=P, thermo_pressure=p, thermo_volume=V,
        stress=ref.stress(), potential_energy=ref.potential_energy(),
        n_rebuilds=np.array([ref.n_rebuilds]))
    ref.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


# One spec frame and one posit frame written by the reference's own
# Filament::WriteSpec / WritePosit after a run (the bytes as written), and
# the global order of that state (Filament::GetPolarOrder / GetNematicOrder).
FORMAT_CASES = {
    "format_3d": dict(n_dim=3, R=15.0, n_fil=12, n_seg=20, lp=500.0, delta=1e-4, seed=31,
                      steps=21),
    "format_2d": dict(n_dim=2, R=20.0, n_fil=16, n_seg=16, lp=20.0, delta=1e-4, seed=32,
                      steps=41),
}


def make_format_case(name, c):
    import tempfile
    nb = np.full(c["n_fil"], c["n_seg"], dtype=np.int32)
    sites = sc.insert_filaments(c["n_dim"], c["R"], c["seed"], nb, nb.astype(float),
                                np.full(c["n_fil"], c["lp"]))
    system = dict(n_dim=c["n_dim"], system_radius=c["R"], delta=c["delta"], seed=c["seed"])
    fils = [dict(length=float(c["n_seg"]), persistence_length=c["lp"], diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * c["n_fil"]
    ref = Reference(system, fils, sites, n_threads=2)
    ref.step(c["steps"])
    with tempfile.TemporaryDirectory() as tmp:
        spec, posit = os.path.join(tmp, "f.spec"), os.path.join(tmp, "f.posit")
        ref.write_spec_frame(spec)
        ref.write_posit_frame(posit)
        spec_b = np.frombuffer(open(spec, "rb").read(), dtype=np.uint8)
        posit_b = np.frombuffer(open(posit, "rb").read(), dtype=np.uint8)
    polar, nematic = ref.global_order()
    out = dict(
        system=np.array([c["n_dim"], c["R"], c["delta"], c["seed"], c["lp"], c["n_seg"],
                         c["n_fil"], c["steps"]], dtype=np.float64),
        sites0=sites, sites=ref.sites(), spec_frame=spec_b, posit_frame=posit_b,
        polar_order=polar, nematic_order=nematic)
    ref.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


# Doubly-bound crosslinks placed, updated and applied by the reference's own
# Crosslink and Anchor code (anchors follow their mesh lambda as the bonds
# stretch, and move between neighbouring bonds), with the tether forces
# recomputed on even steps and re-applied on odd ones.
TETHER_CASES = {
    "tether_3d": dict(n_dim=3, R=10.0, n_fil=20, n_seg=20, lp=50.0, delta=1e-4, seed=41,
                      steps=41, links=0.002, k=10.0, kc=-1.0, rest=1.0),
    "tether_2d": dict(n_dim=2, R=24.0, n_fil=24, n_seg=16, lp=50.0, delta=1e-4, seed=42,
                      steps=41, links=0.002, k=10.0, kc=4.0, rest=1.5),
}


def make_tether_case(name, c):
    from simcore_b200 import workloads
    nb = np.full(c["n_fil"], c["n_seg"], dtype=np.int32)
    sites = sc.insert_filaments(c["n_dim"], c["R"], c["seed"], nb, nb.astype(float),
                                np.full(c["n_fil"], c["lp"]))
    system = dict(n_dim=c["n_dim"], system_radius=c["R"], delta=c["delta"], seed=c["seed"])
    fils = [dict(length=float(c["n_seg"]), persistence_length=c["lp"], diameter=1.0,
                 min_bond_length=0.666, friction_ratio=2.0)] * c["n_fil"]
    a, b, _, _ = workloads.crosslinks("E", sites, fils, 2 * c["R"], scale=c["links"],
                                      seed=c["seed"])
    ref = Reference(system, fils, sites, n_threads=2)
    ref.add_crosslinks(a, b, k_spring=c["k"], k_spring_compress=c["kc"], rest_length=c["rest"])
    ref.step(c["steps"])
    f, t = ref.bond_forces()
    out = dict(
        system=np.array([c["n_dim"], c["R"], c["delta"], c["seed"], c["lp"], c["n_seg"],
                         c["n_fil"], c["steps"]], dtype=np.float64),
        links=np.array([c["k"], c["kc"], c["rest"]]), site_a=a, site_b=b,
        sites0=sites, sites=ref.sites(), prev_sites=ref.prev_sites(), bond_force=f,
        bond_torque=t, tensions=ref.tensions(), crosslink_forces=ref.crosslink_forces(),
        n_rebuilds=np.array([ref.n_rebuilds]))
    ref.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


if __name__ == "__main__":
    # Arguments: the names of the cases to (re)generate; none = all.
    if not Reference.available():
        sys.exit("oracle/_ref/libscref.so is not built (python oracle/build.py)")
    want = set(sys.argv[1:])
    for name, c in CASES.items():
        if want and name not in want:
            continue
        o = make_case(name, c)
        print(name, "rebuilds", int(o["n_rebuilds"][0]), "renormalised filaments",
              int((o["n_normalize"] < c["steps"]).sum()), "pairs", len(o["pairs"]))
    for name, c in THERMO_CASES.items():
        if want and name not in want:
            continue
        o = make_thermo_case(name, c)
        print(name, "rebuilds", int(o["n_rebuilds"][0]), "records", len(o["thermo_step"]))
    for name, c in FORMAT_CASES.items():
        if want and name not in want:
            continue
        o = make_format_case(name, c)
        print(name, "spec bytes", len(o["spec_frame"]), "posit bytes", len(o["posit_frame"]))
    for name, c in TETHER_CASES.items():
        if want and name not in want:
            continue
        o = make_tether_case(name, c)
        print(name, "links", len(o["site_a"]), "max tether force",
              float(np.abs(o["crosslink_forces"]).max()))
