"""Seeded synthetic meshes in openCARP layout (the stand-ins for the private
ventricle/atrium meshes the published TorchCor timings use).

* ``cube``      : structured tetrahedral cube, n elements per edge, each hex
                  split into 6 tets around its v0-v6 diagonal; node index
                  ``(i*(n+1)+j)*(n+1)+k`` for x = i*h, y = j*h, z = k*h.
* ``icosphere`` : subdivided icosahedron projected on a sphere (triangles).

Coordinates are produced in micrometres, the unit ``load_mesh`` divides by
``unit_conversion=1000``; every generator is deterministic for a given seed.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

# the six tetrahedra of a hex cell (corner numbering of ``_HEX``), all sharing
# the v0-v6 diagonal
_HEX = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
_TETS = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]


def cube(n: int, h_mm: float):
    """(nodes_um (N,3) float64, tets (E,4) int64) of an n^3-cell tet cube."""
    g = np.arange(n + 1, dtype=np.float64) * (h_mm * 1000.0)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    corner = [((i + a) * (n + 1) + (j + b)) * (n + 1) + (k + c) for a, b, c in _HEX]
    tets = np.empty((n ** 3, 6, 4), dtype=np.int64)
    for t, quad in enumerate(_TETS):
        for q, v in enumerate(quad):
            tets[:, t, q] = corner[v]
    return nodes, tets.reshape(-1, 4)


def cube_face(n: int, axis: int = 0, side: int = 0):
    """Node indices of one face of the cube (axis 0/1/2, side 0 = low, 1 = high)."""
    idx = np.arange((n + 1) ** 3).reshape(n + 1, n + 1, n + 1)
    sl = [slice(None)] * 3
    sl[axis] = 0 if side == 0 else n
    return np.sort(idx[tuple(sl)].ravel())


def cube_corner_block(n: int, corner, k: int = 5):
    """Node indices of the k x k x k node block at a cube corner in {0,1}^3."""
    rng = [np.arange(k) if c == 0 else np.arange(n + 1 - k, n + 1) for c in corner]
    i, j, l = np.meshgrid(*rng, indexing="ij")
    return np.sort(((i * (n + 1) + j) * (n + 1) + l).ravel())


def pick_corners(seed: int, count: int = 2):
    """``count`` distinct cube corners chosen with ``numpy.random.default_rng(seed)``."""
    corners = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    sel = np.random.default_rng(seed).choice(8, size=count, replace=False)
    return [corners[s] for s in sel]


def centroids(nodes, elems):
    return nodes[elems].mean(axis=1)


def fibres_constant(n_elems: int, direction=(1.0, 0.0, 0.0)):
    return np.tile(np.asarray(direction, dtype=np.float64), (n_elems, 1))


def fibres_rotating_z(nodes_um, elems, angle0_deg=-60.0, angle1_deg=60.0):
    """Fibre angle in the xy-plane varying linearly with the element centroid z."""
    c = centroids(nodes_um, elems)
    z0, z1 = nodes_um[:, 2].min(), nodes_um[:, 2].max()
    th = np.deg2rad(angle0_deg + (angle1_deg - angle0_deg) * (c[:, 2] - z0) / (z1 - z0))
    return np.stack([np.cos(th), np.sin(th), np.zeros_like(th)], 1)


def regions_split_x(nodes_um, elems, ids=(1, 2)):
    """Region ids[0] for centroid x below the mid-plane, ids[1] above."""
    c = centroids(nodes_um, elems)
    mid = 0.5 * (nodes_um[:, 0].min() + nodes_um[:, 0].max())
    return np.where(c[:, 0] < mid, ids[0], ids[1]).astype(np.int64)


def icosphere(level: int, radius_mm: float):
    """(nodes_um (V,3), tris (F,3)) of a level-``level`` subdivided icosahedron."""
    p = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    verts = [np.asarray(x, dtype=np.float64) / np.linalg.norm(x) for x in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.asarray(verts) * (radius_mm * 1000.0)
    return nodes, np.asarray(faces, dtype=np.int64)


def icosphere_fast(level: int, radius_mm: float):
    """``icosphere`` with the subdivision vectorised (same faces and node order:
    new midpoint nodes are numbered in order of their edge's first appearance)."""
    nodes0, faces0 = icosphere(0, 1.0)
    verts = nodes0 / 1000.0
    faces = faces0
    for _ in range(level):
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        e = np.stack([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)], 1).reshape(-1, 2)
        key = np.minimum(e[:, 0], e[:, 1]) * (len(verts) + 1) + np.maximum(e[:, 0], e[:, 1])
        uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        ue = e[first[order]]
        m = verts[ue[:, 0]] + verts[ue[:, 1]]
        m /= np.sqrt((m * m).sum(1))[:, None]
        mid_id = (len(verts) + rank[inv]).reshape(-1, 3)
        ab, bc, ca = mid_id[:, 0], mid_id[:, 1], mid_id[:, 2]
        faces = np.stack([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                          np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3)
        verts = np.concatenate([verts, m])
    return verts * (radius_mm * 1000.0), faces.astype(np.int64)


def fibres_random_tangent(nodes_um, tris, seed: int):
    """Unit fibre per triangle, uniform angle in the plane normal to the centroid."""
    c = centroids(nodes_um, tris)
    nrm = c / np.linalg.norm(c, axis=1, keepdims=True)
    ref = np.where(np.abs(nrm[:, 2:3]) < 0.9, np.array([[0.0, 0.0, 1.0]]), np.array([[1.0, 0.0, 0.0]]))
    e1 = np.cross(nrm, ref)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    e2 = np.cross(nrm, e1)
    th = np.random.default_rng(seed).uniform(0.0, 2.0 * np.pi, size=len(tris))
    return np.cos(th)[:, None] * e1 + np.sin(th)[:, None] * e2


def _fmt_rows(fmt, arr):
    return "".join(fmt % tuple(r) for r in arr)


def write_opencarp(mesh_dir, name, nodes_um, elems, regions, fibres):
    """Write ``name.pts/.elem/.lon`` (openCARP text layout) into ``mesh_dir``."""
    d = Path(mesh_dir)
    os.makedirs(d, exist_ok=True)
    k = elems.shape[1]
    tag = "Tt" if k == 4 else "Tr"
    with open(d / f"{name}.pts", "w") as f:
        f.write(f"{len(nodes_um)}\n")
        np.savetxt(f, nodes_um, fmt="%.6f")
    body = np.concatenate([elems, regions.reshape(-1, 1)], 1)
    with open(d / f"{name}.elem", "w") as f:
        f.write(f"{len(elems)}\n")
        np.savetxt(f, body, fmt=tag + " " + " ".join(["%d"] * (k + 1)))
    with open(d / f"{name}.lon", "w") as f:
        f.write("1\n")
        np.savetxt(f, fibres, fmt="%.8f")


def write_vtx(path, idx):
    """Write a ``.vtx`` stimulus file (count line, type line, one index per line)."""
    idx = np.asarray(idx, dtype=np.int64)
    with open(path, "w") as f:
        f.write(f"{len(idx)}\nintra\n")
        np.savetxt(f, idx, fmt="%d")


def _decimal_roundtrip(a, fmt):
    """float(fmt % x) for every x of ``a``, formatting each distinct value once."""
    a = np.asarray(a, dtype=np.float64)
    u, inv = np.unique(a.ravel(), return_inverse=True)
    r = np.array([float(fmt % x) for x in u], dtype=np.float64)
    return r[inv].reshape(a.shape)


def roundtrip(nodes_um, fibres):
    """The values ``load_mesh`` would read back from the files ``write_opencarp``
    writes (``%.6f`` nodes, ``%.8f`` fibres), for in-memory use."""
    return _decimal_roundtrip(nodes_um, "%.6f"), _decimal_roundtrip(fibres, "%.8f")
