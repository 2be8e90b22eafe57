"""Synthetic monodomain workloads (seeded), built in memory.

``ttp_cube``: ten Tusscher-Panfilov ENDO on an n^3-cell tet cube (default
n=100, h=0.25 mm: 1,030,301 nodes, 6,000,000 tets), fibre angle rotating
linearly from -60 to +60 degrees across z, two conductivity regions split at
the x mid-plane (il/it = 0.5272/0.2076 and 0.9074/0.3332 S/m), two 5x5x5-node
corner blocks stimulated at t = 0 and t = 5 ms (1 ms, intensity 100; the
corners are drawn with numpy.random.default_rng(seed)), dt = 0.01 ms,
T = 100 ms.  It stands in for the private biventricle/slab meshes of the
reference's published timings.

``ms_cube``: Mitchell-Schaeffer on a 20^3-cell cube with 1 mm spacing
(9,261 nodes), fibres along +x, il/it = 0.5/0.2, the x = 0 face stimulated for
1 ms with intensity 100, dt = 0.01 ms, T = 50 ms.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from torchcor_b200 import meshgen


@dataclass
class Workload:
    name: str
    model: str                 # "ms" | "ttp" | "crn"
    nodes_mm: np.ndarray
    elems: np.ndarray
    regions: np.ndarray
    fibres: np.ndarray
    conductivity: list
    stimuli: list              # dicts: region (node ids), start, duration, intensity
    dt: float
    T: float
    cell_type: str = "ENDO"
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self):
        return int(self.nodes_mm.shape[0])

    @property
    def nt(self):
        return int(self.T / self.dt)


def ttp_cube(n=100, h_mm=0.25, seed=1234, T=100.0, dt=0.01):
    nodes_um, tets = meshgen.cube(n, h_mm)
    fib = meshgen.fibres_rotating_z(nodes_um, tets)
    reg = meshgen.regions_split_x(nodes_um, tets)
    stims = [dict(region=meshgen.cube_corner_block(n, c, 5), start=5.0 * k, duration=1.0, intensity=100)
             for k, c in enumerate(meshgen.pick_corners(seed, 2))]
    cond = [dict(region_ids=[1], il=0.5272, it=0.2076), dict(region_ids=[2], il=0.9074, it=0.3332)]
    return Workload(f"ttp_endo_tet_cube_{n}^3_h{h_mm}mm", "ttp", nodes_um / 1000.0, tets, reg, fib, cond, stims,
                    dt, T, meta=dict(n=n, h_mm=h_mm, seed=seed))


def ms_cube(n=20, h_mm=1.0, T=50.0, dt=0.01):
    nodes_um, tets = meshgen.cube(n, h_mm)
    fib = meshgen.fibres_constant(len(tets))
    reg = np.ones(len(tets), dtype=np.int64)
    stims = [dict(region=meshgen.cube_face(n, 0, 0), start=0.0, duration=1.0, intensity=100)]
    cond = [dict(region_ids=[1], il=0.5, it=0.2)]
    return Workload(f"ms_tet_cube_{n}^3_h{h_mm}mm", "ms", nodes_um / 1000.0, tets, reg, fib, cond, stims, dt, T,
                    meta=dict(n=n, h_mm=h_mm))


def cube_face_sim(n, h_mm, model, scale, face, T=100.0, dt=0.01, name=None):
    """One cube of the batched mix: n^3 cells, fibres along +x, conductivity
    scale * (il=0.5, it=0.2), face ``face`` (0..5 = -x,+x,-y,+y,-z,+z) stimulated
    at t = 0 for 1 ms with intensity 100."""
    nodes_um, tets = meshgen.cube(n, h_mm)
    fib = meshgen.fibres_constant(len(tets))
    reg = np.ones(len(tets), dtype=np.int64)
    stims = [dict(region=meshgen.cube_face(n, face // 2, face % 2), start=0.0, duration=1.0, intensity=100)]
    cond = [dict(region_ids=[1], il=0.5 * scale, it=0.2 * scale)]
    return Workload(name or f"{model}_cube_{n}", model, nodes_um / 1000.0, tets, reg, fib, cond, stims, dt, T,
                    meta=dict(n=n, h_mm=h_mm, scale=scale, face=face))


def batch_cubes(count=64, seed=2024, lo=16, hi=64, h_mm=0.25, T=100.0, dt=0.01):
    """``count`` independent cubes: edge length uniform in lo..hi nodes, conductivity
    scale uniform in [0.5, 2], one random face stimulated, Mitchell-Schaeffer and
    ten Tusscher-Panfilov ENDO alternating (50/50), dt 0.01 ms, T 100 ms."""
    rng = np.random.default_rng(seed)
    edges = rng.integers(lo, hi + 1, size=count)
    scales = rng.uniform(0.5, 2.0, size=count)
    faces = rng.integers(0, 6, size=count)
    return [cube_face_sim(int(e) - 1, h_mm, "ms" if k % 2 == 0 else "ttp", float(sc), int(f), T, dt,
                          name=f"cube{k}_{int(e)}nodes_{'ms' if k % 2 == 0 else 'ttp'}")
            for k, (e, sc, f) in enumerate(zip(edges, scales, faces))]


WORKLOADS = {"ttp_cube": ttp_cube, "ms_cube": ms_cube}


def algorithmic_bytes(n_nodes, nnz, n_states):
    """Per-step byte counts of the monodomain step (fp32 values, int32 indices):
    ionic kernel N*(8S+20) (S states incl. V read+written, b' written, AT/RT
    read+written); right-hand side + CG setup 16*nnz + 4(N+1) + 36N; one CG
    iteration 8*nnz + 4(N+1) + 28N."""
    S = n_states + 1
    b_ion = n_nodes * (8 * S + 20)
    b_rhs = 16 * nnz + 4 * (n_nodes + 1) + 36 * n_nodes
    b_iter = 8 * nnz + 4 * (n_nodes + 1) + 28 * n_nodes
    return b_ion, b_rhs, b_iter
