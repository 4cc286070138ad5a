"""The benchmark's CPU-side contract: the reference arm (the reference's own
CPU code on the host cores) prints one JSON line in the shape the GPU arm
prints, and the roofline byte counts follow their stated formulas."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from checkers import Reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Runs the reference arm in-process and then reports whether anything of
# the CUDA library was loaded (module or shared object).
_RUN_REFERENCE_ARM = """
import sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "A", "--steps", "1",
            "--warmup", "3"]
sys.path.insert(0, %r)
import bench
bench.main()
maps = open("/proc/self/maps").read()
print("LOADED", int("simcore_b200" in sys.modules), int("libsimcore_b200" in maps))
"""


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
def test_reference_arm_prints_one_contract_line():
    """One JSON line in the contract's shape, with the GPU arm's `config`,
    and the CUDA library neither imported nor mapped: the arm's inputs come
    from the oracle's insertion."""
    out = subprocess.run([sys.executable, "-c", _RUN_REFERENCE_ARM % ROOT],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert lines[-1] == "LOADED 0 0", lines[-1]
    lines = lines[:-1]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "segment-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.workload_config("A")
    assert d["config"]["workload"].startswith("A:")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_algorithmic_bytes():
    sys.path.insert(0, ROOT)
    import bench
    ns, nb, npairs = 220000, 200000, 124288
    b_int, b_pair = bench.algorithmic_bytes(ns, nb, npairs, "mixed")
    assert b_int == 96 * ns + 56 * nb
    assert b_pair == 56 * nb + 8 * npairs
    b_int, b_pair = bench.algorithmic_bytes(ns, nb, npairs, "fp64")
    assert b_int == 96 * ns + 104 * nb
    assert bench.fused_bytes(ns, nb, npairs) == 96 * ns + 64 * nb + 8 * npairs


@pytest.mark.skipif(not Reference.available(), reason="reference build not present")
def test_tethered_cpu_baseline_runs_the_reference_crosslinks():
    """The CPU baseline of a crosslinked network is the reference's own code,
    its tethers attached by its own Crosslink and Anchor classes, and it
    steps."""
    sys.path.insert(0, ROOT)
    import bench
    from checkers import oracle_workload
    wl = oracle_workload("E", seed=0, scale=0.002)
    assert wl[4] is not None and len(wl[4][0]) > 0
    kind, cores, runs, note = bench.cpu_runs(wl, 2)
    assert kind == "reference" and cores == 2 and len(runs) == 1
    assert "reference" in note
    make, n_bonds = runs[0]
    sim = make()
    try:
        assert sim.n_links == len(wl[4][0])
        assert sim.step(2) >= 0.0
        assert np.isfinite(sim.sites()).all()
    finally:
        sim.close()
