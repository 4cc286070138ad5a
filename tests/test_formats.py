"""The readers of tests/ref_formats.py (which the GPU output tests use on the
library's spec and posit files) against frames written by the reference's
own Filament::WriteSpec and Filament::WritePosit (tests/golden/format_*.npz,
made by tests/golden/make_golden.py): they decode to the oracle's state after
the same steps, so a file the library writes that decodes to its state holds
the reference's bytes.  Likewise the host formula of the global order that
the GPU analysis test checks the device against, against the reference's own
Filament::GetPolarOrder / GetNematicOrder on that state."""
import glob
import os
import struct

import numpy as np
import pytest

from checkers import Oracle
from ref_formats import read_posit, read_spec
from test_oracle import _case

FORMAT_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden",
                                              "format_*.npz")))


def test_format_fixtures_present():
    assert FORMAT_GOLDEN


@pytest.mark.parametrize("path", FORMAT_GOLDEN, ids=[os.path.basename(p) for p in FORMAT_GOLDEN])
def test_reference_written_frames_read_back(path, tmp_path):
    import simcore_b200 as sc
    z, system, fils, steps = _case(path)
    o = Oracle(system, fils, z["sites0"])
    o.step(steps)
    xyz = o.sites()
    o.close()
    assert np.array_equal(xyz, z["sites"])
    # File header (SpeciesBase::InitSpecFileOutput order: n_steps, cadence,
    # delta), then the frame as the reference wrote it.
    head = struct.pack("<iid", steps, 1, system["delta"])
    (tmp_path / "f.spec").write_bytes(head + z["spec_frame"].tobytes())
    (tmp_path / "f.posit").write_bytes(head + z["posit_frame"].tobytes())
    nb = np.array([sc.filament_n_bonds(f) for f in fils])
    off = np.concatenate([[0], np.cumsum(nb + 1)])

    h, frames = read_spec(str(tmp_path / "f.spec"))
    assert h == (steps, 1, system["delta"]) and len(frames) == 1 and len(frames[0]) == len(fils)
    for k, rec in enumerate(frames[0]):
        assert np.array_equal(rec["sites"], xyz[off[k]:off[k + 1]])
        assert rec["diameter"] == fils[k]["diameter"] and rec["length"] == fils[k]["length"]
        assert rec["bond_length"] == fils[k]["length"] / nb[k]
        assert rec["bending_stiffness"] == fils[k]["persistence_length"] and rec["poly"] == 0

    h, pframes = read_posit(str(tmp_path / "f.posit"))
    assert len(pframes) == 1 and pframes[0].shape == (len(fils), 11)
    R = system["system_radius"]
    for k, rec in enumerate(pframes[0]):
        s = xyz[off[k]:off[k + 1]]
        p = np.zeros(3)
        for v in s:
            p = p + v
        p = p / len(s)
        assert np.array_equal(rec[0:3], p)
        d = s[1:] - s[:-1]
        u = d / np.sqrt((d * d).sum(axis=1))[:, None]
        a = np.zeros(3)
        for v in list(u) + [u[-1]]:
            a = a + v
        a = a / np.sqrt((a * a).sum())
        assert np.abs(rec[6:9] - a).max() < 1e-14
        s_img = p / (2 * R)
        s_img -= np.where(s_img < 0, np.ceil(s_img - 0.5), np.floor(s_img + 0.5))
        assert np.abs(rec[3:6] - s_img).max() < 1e-14
        assert rec[9] == fils[k]["diameter"] and rec[10] == fils[k]["length"]


@pytest.mark.parametrize("path", FORMAT_GOLDEN, ids=[os.path.basename(p) for p in FORMAT_GOLDEN])
def test_global_order_formula_matches_reference(path):
    """The mean over filaments of the mean bond orientation and of the bond
    tensor (2 u u^T - I), n_dim x n_dim in a 3 x 3 array, from the bond
    orientations of the final sites: the reference's values to 1e-12."""
    import simcore_b200 as sc
    z, system, fils, steps = _case(path)
    nd = system["n_dim"]
    xyz = z["sites"]
    nb = np.array([sc.filament_n_bonds(f) for f in fils])
    off = np.concatenate([[0], np.cumsum(nb + 1)])
    pv = np.zeros(3)
    q = np.zeros((3, 3))
    for k in range(len(fils)):
        s = xyz[off[k]:off[k + 1], :nd]
        d = s[1:] - s[:-1]
        u = d / np.sqrt((d * d).sum(axis=1))[:, None]
        pv[:nd] += u.mean(0)
        q[:nd, :nd] += (2 * np.einsum("bi,bj->ij", u, u) - len(u) * np.eye(nd)) / len(u)
    pv /= len(fils)
    q /= len(fils)
    assert np.abs(pv - z["polar_order"]).max() < 1e-12
    assert np.abs(q - z["nematic_order"]).max() < 1e-12
    assert np.abs(z["nematic_order"]).max() > 0.05  # not a trivial state
