"""The library's spec output byte for byte against a frame written by the
reference's own Filament::WriteSpec (tests/golden/format_3d.npz): the FP64
path reaches the reference's state after the same steps, so the frame it
writes holds the same bytes.  The posit frame's orientation and scaled
position come from the device's averages, whose rounding differs: they are
compared as numbers."""
import os
import struct

import numpy as np
import pytest

from ref_formats import read_posit
from test_oracle import _case

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "format_3d.npz")


def test_spec_frame_is_the_references_bytes(tmp_path):
    import simcore_b200 as sc
    z, system, fils, steps = _case(FIXTURE)
    ctx = sc.Context(system, fils, z["sites0"], precision="fp64")
    run = str(tmp_path / "fmt")
    ctx.output_open(run, n_steps=steps, n_posit=steps, n_spec=steps)
    ctx.output_write()  # step 0
    ctx.step(steps)
    ctx.output_write()  # step `steps`
    ctx.output_close()
    ctx.close()
    spec = open(run + "_filament_filament.spec", "rb").read()
    want = z["spec_frame"].tobytes()
    assert spec[:16] == struct.pack("<iid", steps, steps, system["delta"])
    assert len(spec) == 16 + 2 * len(want)
    assert spec[16 + len(want):] == want

    posit = open(run + "_filament_filament.posit", "rb").read()
    ref = z["posit_frame"].tobytes()
    assert len(posit) == 16 + 2 * len(ref)
    (tmp_path / "ref.posit").write_bytes(posit[:16] + ref)
    _, ours = read_posit(run + "_filament_filament.posit")
    _, theirs = read_posit(str(tmp_path / "ref.posit"))
    a, b = ours[1], theirs[0]
    assert np.array_equal(a[:, 0:3], b[:, 0:3])      # average positions
    assert np.abs(a[:, 3:9] - b[:, 3:9]).max() < 1e-13
    assert np.array_equal(a[:, 9:11], b[:, 9:11])    # diameter, length
