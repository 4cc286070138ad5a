"""Readers of the reference's binary output files, written from its own
readers, for checking that GPU runs can be read back by the reference's
analyses.

spec file (SpeciesBase::InitSpecFileInput, src/species_base.cpp:55-70 for the
header; Species::ReadSpecs, include/simcore/species.hpp:233-258; Mesh::ReadSpec
and Filament::ReadSpec, src/mesh.cpp:482-492, src/filament.cpp:1330-1337):
  int n_steps, int n_spec, double delta, then per frame int n_members and per
  filament double diameter, length, bond_length, int n_sites,
  double[3 n_sites] positions, double bending_stiffness, uchar poly.
posit file (SpeciesBase::InitPositFileInput, src/species_base.cpp:29-45;
Filament::WritePosit, src/filament.cpp:1345-1361):
  int n_steps, int n_posit, double delta, then per frame int n_members and per
  filament double[3] avg_pos, double[3] avg_scaled_pos, double[3] avg_u,
  double diameter, double length.
"""
import struct

import numpy as np


def _header(f):
    n_steps, cadence = struct.unpack("<ii", f.read(8))
    (delta,) = struct.unpack("<d", f.read(8))
    return n_steps, cadence, delta


def read_spec(path):
    frames = []
    with open(path, "rb") as f:
        head = _header(f)
        while True:
            raw = f.read(4)
            if len(raw) < 4:
                break
            (n,) = struct.unpack("<i", raw)
            fils = []
            for _ in range(n):
                diam, length, bl = struct.unpack("<ddd", f.read(24))
                (ns,) = struct.unpack("<i", f.read(4))
                pos = np.frombuffer(f.read(24 * ns), dtype="<f8").reshape(ns, 3).copy()
                (kappa,) = struct.unpack("<d", f.read(8))
                (poly,) = struct.unpack("<B", f.read(1))
                fils.append(dict(diameter=diam, length=length, bond_length=bl, sites=pos,
                                 bending_stiffness=kappa, poly=poly))
            frames.append(fils)
    return head, frames


def read_posit(path):
    frames = []
    with open(path, "rb") as f:
        head = _header(f)
        while True:
            raw = f.read(4)
            if len(raw) < 4:
                break
            (n,) = struct.unpack("<i", raw)
            rec = np.frombuffer(f.read(88 * n), dtype="<f8").reshape(n, 11).copy()
            frames.append(rec)
    return head, frames
