"""Inputs of the golden cases: meshes, conductivities, stimuli, ionic inputs.

Shared by ``make_golden.py`` (which runs the reference on them) and the tests
(which rebuild the same inputs for the oracle and the CUDA path).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from torchcor_b200 import meshgen

_STEP = dict(kind="step", dt=0.01, n=4096, seed=3)
_ONE = [dict(region_ids=[1], il=0.5, it=0.2)]
_FACE = [dict(file="face.vtx", nodes=dict(type="face", axis=0, side=0), start=0.0, duration=1.0, intensity=100)]
_TTP_COND = [dict(region_ids=[1], il=0.5272, it=0.2076), dict(region_ids=[2], il=0.9074, it=0.3332)]
_TTP_STIM = [dict(file="c0.vtx", nodes=dict(type="corner", k=3, seed=7, which=0), start=0.0, duration=1.0, intensity=100),
             dict(file="c1.vtx", nodes=dict(type="corner", k=3, seed=7, which=1), start=5.0, duration=1.0, intensity=100)]
_ICO = dict(type="ico", level=3, radius=5.0, fibres="tangent", seed=11)
_ICO_STIM = [dict(file="cap.vtx", nodes=dict(type="zcap", frac=0.9), start=0.0, duration=2.0, intensity=50)]

CASES = [
    # small tet cube, Mitchell-Schaeffer, full matrices and first steps kept
    dict(kind="tissue", name="cube6_ms_f32", model="ms", dtype="f32",
         mesh=dict(type="cube", n=6, h=1.0, fibres="x", regions="one"), conductivity=_ONE, stimuli=_FACE,
         dt=0.01, T=10.0, tol=1e-5, max_iter=100, full_matrices=True, keep_steps=5, keep_states=True),
    # the 20^3 cube, Mitchell-Schaeffer (the reference's CPU-runnable configuration)
    dict(kind="tissue", name="cfg1_ms_f32", model="ms", dtype="f32",
         mesh=dict(type="cube", n=20, h=1.0, fibres="x", regions="one"), conductivity=_ONE, stimuli=_FACE,
         dt=0.01, T=50.0, tol=1e-5, max_iter=100, snapshots=[0, 5, 10, 20, 30, 40, 50], keep_states=True),
    dict(kind="tissue", name="cfg1_ms_f64", model="ms", dtype="f64",
         mesh=dict(type="cube", n=20, h=1.0, fibres="x", regions="one"), conductivity=_ONE, stimuli=_FACE,
         dt=0.01, T=50.0, tol=1e-5, max_iter=100, snapshots=[0, 5, 10, 20, 30, 40, 50]),
    # ten Tusscher-Panfilov on a small cube with the 100^3 case's structure
    dict(kind="tissue", name="cube8_ttp_f32", model="ttp", cell_type="ENDO", dtype="f32",
         mesh=dict(type="cube", n=8, h=0.25, fibres="rotz", regions="splitx"), conductivity=_TTP_COND,
         stimuli=_TTP_STIM, dt=0.01, T=30.0, tol=1e-5, max_iter=100, full_matrices=True, keep_states=True),
    dict(kind="tissue", name="cube8_ttp_f64", model="ttp", cell_type="ENDO", dtype="f64",
         mesh=dict(type="cube", n=8, h=0.25, fibres="rotz", regions="splitx"), conductivity=_TTP_COND,
         stimuli=_TTP_STIM, dt=0.01, T=30.0, tol=1e-5, max_iter=100),
    # Courtemanche on an icosphere shell (triangles)
    dict(kind="tissue", name="ico3_crn_f32", model="crn", dtype="f32", mesh=_ICO,
         conductivity=[dict(region_ids=[1], il=0.4, it=0.1)], stimuli=_ICO_STIM,
         dt=0.02, T=40.0, tol=1e-5, max_iter=100, full_matrices=True, keep_states=True),
    dict(kind="tissue", name="ico3_crn_f64", model="crn", dtype="f64", mesh=_ICO,
         conductivity=[dict(region_ids=[1], il=0.4, it=0.1)], stimuli=_ICO_STIM,
         dt=0.02, T=40.0, tol=1e-5, max_iter=100),
    # intra/extra conductivities (harmonic mean), periodic stimulus with a count
    dict(kind="tissue", name="cube4_ms_period_f32", model="ms", dtype="f32",
         mesh=dict(type="cube", n=4, h=0.5, fibres="x", regions="one"),
         conductivity=[dict(region_ids=[1], il=0.17, it=0.019, el=0.62, et=0.2)],
         stimuli=[dict(file="face.vtx", nodes=dict(type="face", axis=2, side=1), start=0.0, duration=1.0,
                       intensity=100, period=4.0, count=2)],
         dt=0.01, T=12.0, tol=1e-5, max_iter=100, full_matrices=True, phie=True),
    # long enough for repolarisation times (RT) to be set
    dict(kind="tissue", name="cube4_ms_rt_f32", model="ms", dtype="f32",
         mesh=dict(type="cube", n=4, h=0.5, fibres="x", regions="one"), conductivity=_ONE, stimuli=_FACE,
         dt=0.02, T=450.0, tol=1e-5, max_iter=100, snapshots=[0, 1, 2, 100, 200, 400, 450], keep_states=True),
    # per-node TTP conductances set after initialize() and stepped through Monodomain.step
    # (the reference's solve() re-initialises them to uniform values)
    dict(kind="step_api", name="cube8_ttp_nodecond_f32", model="ttp", cell_type="ENDO", dtype="f32",
         mesh=dict(type="cube", n=8, h=0.25, fibres="rotz", regions="splitx"), conductivity=_TTP_COND,
         stimuli=_TTP_STIM, dt=0.01, T=30.0, tol=1e-5, max_iter=100, every=100,
         node_cond=dict(GKs=(0.1, 0.4), Gto=(0.3, 0.05), GKr=(0.1, 0.2), GCaL=(3e-5, 5e-5))),
    # one differentiate() on seeded random inputs spanning the lookup-table ranges
    dict(_STEP, name="step_ms_f32", model="ms", dtype="f32"),
    dict(_STEP, name="step_ttp_f32", model="ttp", cell_type="ENDO", dtype="f32"),
    dict(_STEP, name="step_ttp_epi_f32", model="ttp", cell_type="EPI", dtype="f32"),
    dict(_STEP, name="step_crn_f32", model="crn", dtype="f32", dt=0.02),
    dict(_STEP, name="step_ttp_f64", model="ttp", cell_type="ENDO", dtype="f64"),
    dict(_STEP, name="step_crn_f64", model="crn", dtype="f64", dt=0.02),
    # single-cell action potentials
    dict(kind="cell", name="cell_ms_f32", model="ms", dtype="f32", dt=0.01, T=400.0, every=1.0,
         stim=50.0, stim_start=0.0, stim_dur=2.0),
    dict(kind="cell", name="cell_ttp_f32", model="ttp", cell_type="EPI", dtype="f32", dt=0.02, T=400.0,
         every=1.0, stim=20.0, stim_start=0.0, stim_dur=2.0),
    dict(kind="cell", name="cell_crn_f32", model="crn", dtype="f32", dt=0.02, T=400.0, every=1.0,
         stim=50.0, stim_start=0.0, stim_dur=2.0),
]

# Full-size runs of the benchmark workloads, stored compactly (``compact``):
# activation/repolarisation times as step indices for every node, Vm at a few
# frames on a seeded node sample plus per-frame statistics of every node, the
# CSR pattern as a SHA-256 digest, per-step CG iteration counts.  They take
# tens of minutes of reference CPU time each and are generated on request
# (``make_golden.py --only <name>``).
_CFG2 = dict(kind="tissue", model="ttp", cell_type="ENDO",
             mesh=dict(type="cube", n=100, h=0.25, fibres="rotz", regions="splitx"), conductivity=_TTP_COND,
             stimuli=[dict(file="c0.vtx", nodes=dict(type="corner", k=5, seed=1234, which=0), start=0.0,
                           duration=1.0, intensity=100),
                      dict(file="c1.vtx", nodes=dict(type="corner", k=5, seed=1234, which=1), start=5.0,
                           duration=1.0, intensity=100)],
             dt=0.01, T=40.0, tol=1e-5, max_iter=100, big=True,
             compact=dict(seed=5, vm_sample=32768, vm_frames=[1, 2, 5, 6, 10, 20, 30, 40]))
_CFG3 = dict(kind="tissue", model="crn", mesh=dict(type="ico", level=7, radius=25.0, fibres="tangent", seed=7),
             conductivity=[dict(region_ids=[1], il=0.4, it=0.1)],
             stimuli=[dict(file="cap.vtx", nodes=dict(type="zcap", frac=0.98), start=0.0, duration=2.0,
                           intensity=50)],
             dt=0.02, T=400.0, tol=1e-5, max_iter=100, big=True,
             compact=dict(seed=5, vm_sample=32768, vm_frames=[1, 2, 4, 10, 50, 100, 200, 300, 350, 400]))

BIG_CASES = [
    # TTP ENDO on the 100^3-cell cube (1,030,301 nodes): the single-simulation benchmark workload
    # over its first 40 ms (4,000 steps: both stimuli, the fronts crossing the cube)
    dict(_CFG2, name="cfg2_ttp_f32", dtype="f32"),
    dict(_CFG2, name="cfg2_ttp_f64", dtype="f64"),
    # CRN on the level-7 icosphere (163,842 nodes), run through repolarisation (T = 400 ms)
    dict(_CFG3, name="cfg3_crn_f32", dtype="f32"),
    dict(_CFG3, name="cfg3_crn_f64", dtype="f64"),
]


def case(name):
    for c in CASES + BIG_CASES:
        if c["name"] == name:
            return c
    raise KeyError(name)


def mesh_arrays(case):
    """(nodes_um, elems, regions, fibres) of a tissue case, before file output."""
    m = case["mesh"]
    if m["type"] == "cube":
        nodes, elems = meshgen.cube(m["n"], m["h"])
        if m["fibres"] == "x":
            fib = meshgen.fibres_constant(len(elems))
        else:
            fib = meshgen.fibres_rotating_z(nodes, elems)
        if m["regions"] == "one":
            reg = np.ones(len(elems), dtype=np.int64)
        else:
            reg = meshgen.regions_split_x(nodes, elems)
    else:
        nodes, elems = meshgen.icosphere(m["level"], m["radius"])
        fib = meshgen.fibres_random_tangent(nodes, elems, m["seed"])
        reg = np.ones(len(elems), dtype=np.int64)
    return nodes, elems, reg, fib


def stimulus_nodes(case, spec, nodes_um):
    m = case["mesh"]
    if spec["type"] == "face":
        return meshgen.cube_face(m["n"], spec["axis"], spec["side"])
    if spec["type"] == "corner":
        corner = meshgen.pick_corners(spec["seed"], 2)[spec["which"]]
        return meshgen.cube_corner_block(m["n"], corner, spec["k"])
    if spec["type"] == "zcap":
        return np.nonzero(nodes_um[:, 2] > spec["frac"] * m["radius"] * 1000.0)[0]
    raise ValueError(spec)


def write_case_mesh(case, mesh_dir):
    """Write the case's mesh and ``.vtx`` files into ``mesh_dir``."""
    nodes, elems, reg, fib = mesh_arrays(case)
    meshgen.write_opencarp(mesh_dir, "mesh", nodes, elems, reg, fib)
    for s in case["stimuli"]:
        meshgen.write_vtx(Path(mesh_dir) / s["file"], stimulus_nodes(case, s["nodes"], nodes))


TTP_INIT = dict(CaSR=1.3, CaSS=0.00007, Cai=0.00007, Ki=138.3, Nai=7.67, R_=1.0)
TTP_GATES = ["D", "F", "F2", "FCaSS", "H", "J", "M", "R", "S", "Xr1", "Xr2", "Xs"]
CRN_INIT = dict(Ca_rel=1.49, Ca_up=1.49, Cai=1.02e-1, Ki=139.0)
CRN_GATES = ["d", "f", "f_Ca", "h", "j", "m", "oa", "oi", "u", "ua", "ui", "v", "w", "xr", "xs"]


def random_ionic_inputs(case):
    """Seeded V and state arrays spanning the table ranges (plus exact edges)."""
    rng = np.random.default_rng(case["seed"])
    n = case["n"]
    edges = np.array([-900.0, -800.0, -200.0, -100.0, -47.13, -40.0, -10.0, 0.0, 7.9, 15.0, 200.0,
                      799.99, 800.0, 900.0])
    V = rng.uniform(-110.0, 70.0, size=n)
    V[:len(edges)] = edges
    st = {}
    if case["model"] == "ms":
        st["H"] = rng.uniform(0.0, 1.0, size=n)
    elif case["model"] == "ttp":
        for k, v in TTP_INIT.items():
            st[k] = v * np.exp(rng.normal(0.0, 0.4, size=n))
        st["R_"] = rng.uniform(0.0, 1.0, size=n)
        for g in TTP_GATES:
            st[g] = rng.uniform(0.0, 1.0, size=n)
    else:
        for k, v in CRN_INIT.items():
            st[k] = v * np.exp(rng.normal(0.0, 0.4, size=n))
        for g in CRN_GATES:
            st[g] = rng.uniform(0.0, 1.0, size=n)
    dt = np.float64 if case["dtype"] == "f64" else np.float32
    return V.astype(dt), {k: v.astype(dt) for k, v in st.items()}


def node_values(lo, hi, n):
    """Per-node parameter values rising linearly with the node index (float32)."""
    return (lo + (hi - lo) * np.arange(n, dtype=np.float64) / max(n - 1, 1)).astype(np.float32)
