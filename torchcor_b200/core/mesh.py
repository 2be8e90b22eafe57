"""openCARP mesh reader with the behaviour of ``torchcor/core/mesh.py:5-63``.

Same files (``.pts`` header + coordinates, ``.elem`` header + ``Tt``/``Tr``
rows with a trailing region id, ``.lon`` header + one fibre per element), same
unit conversion and the same ``ValueError`` on count mismatches.  Parsing uses
pandas' C tokenizer with round-trip float conversion, which reads the same
doubles as ``np.loadtxt`` at a fraction of the time on large meshes.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pandas as pd


def _table(path, usecols=None, dtype=None):
    df = pd.read_csv(path, sep=r"\s+", header=None, skiprows=1, usecols=usecols, dtype=dtype,
                     float_precision="round_trip", engine="c")
    return np.ascontiguousarray(df.to_numpy())


class MeshReader:
    def __init__(self, mesh_dir: str):
        self.mesh_dir = Path(mesh_dir)
        self.node_file = self.elem_file = self.fibre_file = None
        for p in self.mesh_dir.iterdir():
            if p.suffix == ".pts":
                self.node_file = p
            elif p.suffix == ".elem":
                self.elem_file = p
            elif p.suffix == ".lon":
                self.fibre_file = p
        self.nodes = self.elems = self.regions = self.fibres = None

    def read_nodes(self, unit_conversion=1000):
        with self.node_file.open("r") as f:
            expected = int(f.readline().strip())
        nodes = _table(self.node_file, dtype=np.float64)
        if nodes.shape[0] != expected:
            raise ValueError(f"Mismatch in number of nodes: expected {expected}, but found {nodes.shape[0]}")
        self.nodes = nodes / unit_conversion

    def read_elems(self):
        with self.elem_file.open("r") as f:
            expected = int(f.readline().strip())
            first = f.readline().strip().split()
        usecols = list(range(1, len(first)))
        data = _table(self.elem_file, usecols=usecols, dtype=np.int64)
        if data.shape[0] != expected:
            raise ValueError(f"Mismatch: expected {expected}, but found {data.shape[0]}")
        self.elems = data[:, :-1]
        self.regions = data[:, -1]

    def read_fibres(self):
        self.fibres = _table(self.fibre_file, dtype=np.float64)

    def read(self, unit_conversion=1000):
        self.read_nodes(unit_conversion)
        self.read_elems()
        self.read_fibres()
        return self.nodes, self.elems, self.regions, self.fibres


def read_vtx(vtx_filepath):
    """Node indices of a ``.vtx`` file (count line, type line, indices), as
    ``Stimuli.load_stimulus_region`` (stimulation.py:20-29)."""
    with Path(vtx_filepath).open("r") as f:
        size = int(f.readline().strip())
    region = np.loadtxt(vtx_filepath, dtype=int, skiprows=2, ndmin=1)
    if len(region) != size:
        raise Exception(f"Error loading {vtx_filepath}")
    return region.astype(np.int64)
