"""The C++ host classes (include/simcore_host.hpp): Simulation,
InteractionManager and FilamentSpecies keep the reference's names and roles
and call the C ABI.  A C++ program compiled against the headers and linked
with the library (tests/native/host_classes_run.cpp) runs the reference's
step loop -- host-driven steps with a per-step hook, then captured steps --
and must give the bits the Python binding gives for the same calls."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "host_classes_run.cpp")


def _build(tmp_path):
    """Compiles the program against include/ and links libsimcore_b200.so."""
    cxx = shutil.which("g++") or "/usr/bin/g++"
    exe = str(tmp_path / "host_classes_run")
    lib_dir = os.path.join(ROOT, "simcore_b200")
    cmd = [cxx, "-std=c++14", "-O2", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L" + lib_dir, "-lsimcore_b200", "-Wl,-rpath," + lib_dir]
    subprocess.check_call(cmd)
    return exe


def test_host_classes_compile_and_link(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_classes_match_python_binding(tmp_path, precision):
    import simcore_b200 as sc
    from simcore_b200 import workloads
    exe = _build(tmp_path)
    system, fils, sites = workloads.make("B", 0.02, seed=31)
    n_host, n_graph = 7, 40
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        np.array([system["n_dim"], len(fils), len(sites), 1 if precision == "mixed" else 0],
                 dtype=np.int32).tofile(f)
        np.array([system["system_radius"], system["delta"], system["seed"]]).tofile(f)
        np.array([[q["length"], q["persistence_length"], q["diameter"], q["min_bond_length"],
                   q["friction_ratio"]] for q in fils]).tofile(f)
        np.ascontiguousarray(sites, dtype=np.float64).tofile(f)
    subprocess.check_call([exe, inp, outp, str(n_host), str(n_graph)])
    ctx = sc.Context(system, fils, sites, precision=precision)
    ctx.step(n_host)
    ctx.step_graph(n_graph)
    ctx.interact()
    want_sites = ctx.sites()
    want_f, want_t = ctx.bond_forces()
    rebuilds = ctx.counters().n_rebuilds
    ctx.close()
    raw = np.fromfile(outp, dtype=np.float64, count=3 * len(sites) + 6 * len(want_f))
    ns, nb = 3 * len(sites), 3 * len(want_f)
    assert np.array_equal(raw[:ns].reshape(-1, 3), want_sites)
    assert np.array_equal(raw[ns:ns + nb].reshape(-1, 3), want_f)
    assert np.array_equal(raw[ns + nb:].reshape(-1, 3), want_t)
    tail = np.fromfile(outp, dtype=np.int64)[-1]
    assert tail == rebuilds > 0
