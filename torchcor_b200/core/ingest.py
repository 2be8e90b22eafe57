"""openCARP mesh files read on the device (the role of ``torchcor/core/mesh.py:26-63``).

The bytes of each file go to the GPU once; the newline positions and the
fields are found there (``tcb_text_newlines`` / ``tcb_text_parse``), numbers are
converted with correct rounding, so the arrays equal the host reader's
(``MeshReader``, which reads the doubles ``np.loadtxt`` reads).  A file the
device parser cannot take exactly (a field with more than 19 significant digits
or an exponent beyond its exact range, blank lines inside the table, a row with
a different number of fields, a count that does not match the header) is read
by ``MeshReader`` instead, which also raises the reference's errors.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import torch

from torchcor_b200 import _lib
from torchcor_b200._lib import check, ptr, stream_ptr
from torchcor_b200.core.mesh import MeshReader


class TextTable:
    """A text file on the device with its newline positions."""

    def __init__(self, path, device):
        self.path = Path(path)
        raw = np.fromfile(self.path, dtype=np.uint8)
        self.n = int(raw.size)
        self.text = torch.from_numpy(raw).pin_memory().to(device, non_blocking=True)
        lib = _lib.load()
        scratch = torch.empty(int(lib.tcb_text_scratch(max(self.n, 1))), device=device, dtype=torch.int64)
        cnt = C.c_int64()
        check(lib.tcb_text_newlines(ptr(self.text), self.n, ptr(scratch), None, 0, C.byref(cnt), stream_ptr()))
        self.nl = torch.empty(max(cnt.value, 1), device=device, dtype=torch.int64)
        check(lib.tcb_text_newlines(ptr(self.text), self.n, ptr(scratch), ptr(self.nl), cnt.value, C.byref(cnt),
                                    stream_ptr()))
        self.n_nl = cnt.value
        ends_nl = self.n > 0 and raw[-1] == ord("\n")
        self.n_lines = self.n_nl + (0 if ends_nl else 1)
        with self.path.open("r") as f:
            self.head = [f.readline() for _ in range(2)]

    def parse(self, first_line, rows, skip, cols, as_int):
        """(rows, cols) int64 or float64 device tensor, or None if not exactly parseable."""
        dev = self.text.device
        out = torch.empty((rows, cols), device=dev, dtype=torch.int64 if as_int else torch.float64)
        bad = torch.zeros(1, device=dev, dtype=torch.int64)
        check(_lib.load().tcb_text_parse(ptr(self.text), self.n, ptr(self.nl), self.n_nl, first_line, rows, skip,
                                         cols, int(bool(as_int)), ptr(out), ptr(bad), stream_ptr()))
        return None if int(bad.item()) else out


def read_mesh_device(mesh_dir, device, unit_conversion=1000):
    """(nodes, elems, regions, fibres) as device tensors (float64 nodes already divided
    by ``unit_conversion``, int64 elements and regions, float64 fibres) and the
    list of files that had to be read on the host."""
    host = MeshReader(mesh_dir)
    on_host = []

    # nodes: header count, then x y z per line
    t = TextTable(host.node_file, device)
    expected = int(t.head[0].strip())
    nodes = None
    if t.n_lines - 1 == expected and expected > 0:
        nodes = t.parse(1, expected, 0, len(t.head[1].split()), False)
    if nodes is None:
        host.read_nodes(unit_conversion)
        nodes = torch.from_numpy(host.nodes).to(device)
        on_host.append(host.node_file.name)
    else:
        # float64 division, correctly rounded as numpy's (a tensor divisor: PyTorch
        # turns division by a Python scalar into a multiplication by its reciprocal)
        nodes = nodes / torch.full_like(nodes, float(unit_conversion))
    del t

    # elements: header count, then "Tt a b c d region" / "Tr a b c region"
    t = TextTable(host.elem_file, device)
    expected = int(t.head[0].strip())
    ncols = len(t.head[1].split()) - 1
    data = None
    if t.n_lines - 1 == expected and expected > 0:
        data = t.parse(1, expected, 1, ncols, True)
    if data is None:
        host.read_elems()
        elems = torch.from_numpy(np.ascontiguousarray(host.elems)).to(device)
        regions = torch.from_numpy(np.ascontiguousarray(host.regions)).to(device)
        on_host.append(host.elem_file.name)
    else:
        elems, regions = data[:, :-1].contiguous(), data[:, -1].contiguous()
    del t

    # fibres: header line, then one or more directions per element
    t = TextTable(host.fibre_file, device)
    rows = t.n_lines - 1
    fib = t.parse(1, rows, 0, len(t.head[1].split()), False) if rows > 0 else None
    if fib is None:
        host.read_fibres()
        fib = torch.from_numpy(np.ascontiguousarray(host.fibres)).to(device)
        on_host.append(host.fibre_file.name)
    return nodes, elems, regions, fib, on_host
