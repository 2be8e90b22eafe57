"""Generate the golden fixtures in this directory by running the TorchCor
reference itself (pure Python/PyTorch, CPU).

Run from the repository root, pointing at a TorchCor checkout (``--ref`` or
the ``TORCHCOR_REF`` environment variable):

    python tests/golden/make_golden.py --ref <torchcor checkout> [--only name ...]

The full-size cases (``cases.BIG_CASES``: the 1,030,301-node TTP cube and the
level-7 CRN icosphere, each in float32 and float64) take tens of minutes of
CPU time each and run only when named with ``--only``.

The reference is imported with small stubs for its post-processing imports
(pyvista, matplotlib, the ECG module) and with NVML/``torch.cuda`` calls in
``Monodomain.__init__`` replaced by no-ops, so that ``Monodomain`` runs on a
CPU-only machine.  Meshes come from ``torchcor_b200.meshgen`` and are written
in openCARP text layout, so the reference reads them through its own
``load_mesh``.  Each case writes ``<name>.npz``; ``cases.json`` records the
inputs of every case so the tests can rebuild them without the reference.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import tempfile
import time
import types
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from torchcor_b200 import meshgen  # noqa: E402
from tests.golden import cases as C  # noqa: E402


def import_reference(ref_root):
    sys.path.insert(0, str(ref_root))
    for name in ["pyvista", "matplotlib", "matplotlib.pyplot", "matplotlib.animation"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    ecg = types.ModuleType("torchcor.signalanalysis.signalanalysis.ecg_QS")
    ecg.Ecg = None
    sys.modules["torchcor.signalanalysis.signalanalysis.ecg_QS"] = ecg
    torch.cuda.current_device = lambda: 0
    import torchcor.simulator.monodomain as md

    class _U:
        gpu = 0
        used = 0

    md.nvmlInit = lambda: None
    md.nvmlDeviceGetHandleByIndex = lambda i: None
    md.nvmlDeviceGetUtilizationRates = lambda h: _U()
    md.nvmlDeviceGetMemoryInfo = lambda h: _U()
    import torchcor.ionic as ionic
    return md, ionic


def make_ionic(ionic, model, dt, dtype, params):
    cpu = torch.device("cpu")
    if model == "ms":
        m = ionic.ModifiedMS2v(dt, device=cpu, dtype=dtype)
    elif model == "ttp":
        m = ionic.TenTusscherPanfilov(params.get("cell_type", "ENDO"), dt, device=cpu, dtype=dtype)
    elif model == "crn":
        m = ionic.CourtemancheRamirezNattel(dt, device=cpu, dtype=dtype)
    else:
        raise ValueError(model)
    for k, v in params.get("set", {}).items():
        setattr(m, k, v)
    return m


def run_tissue(md, ionic, case, workdir):
    """One ``Monodomain.solve`` of a tissue case; returns the fixture dict."""
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    mesh_dir = Path(workdir) / case["name"]
    C.write_case_mesh(case, mesh_dir)
    im = make_ionic(ionic, case["model"], case["dt"], dtype, case)
    sim = md.Monodomain(im, T=case["T"], dt=case["dt"], device=torch.device("cpu"), dtype=dtype)
    sim.load_mesh(mesh_dir)
    for cond in case["conductivity"]:
        sim.add_conductivity(**cond)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"], period=s.get("period"), count=s.get("count", 1))
    iters = []
    orig_step = sim.step
    traj = []
    step_wall = []

    def step(u, t, a_tol, r_tol, max_iter, verbose=False):
        t0 = time.perf_counter()
        out = orig_step(u, t, a_tol, r_tol, max_iter, verbose)
        step_wall.append(time.perf_counter() - t0)
        iters.append(out[1])
        if len(traj) < case.get("keep_steps", 0):
            traj.append(out[0].clone())
        if case.get("big") and len(iters) % 500 == 0:
            print(f"  {case['name']}: step {len(iters)}, t={t:.2f}, {np.mean(step_wall[-500:]) * 1e3:.1f} ms/step, "
                  f"{sum(iters)} CG iterations", flush=True)
        return out

    sim.step = step
    out_dir = Path(workdir) / (case["name"] + "_out")
    t0 = time.time()
    total = sim.solve(a_tol=case["tol"], r_tol=case["tol"], max_iter=case["max_iter"], calculate_AT_RT=True,
                      linear_guess=True, snapshot_interval=1, verbose=False, result_path=str(out_dir))
    wall = time.time() - t0
    if case.get("phie"):
        # extracellular potential recovery from the saved Vm frames (monodomain.py:254-286)
        sim.phie_recovery(a_tol=case["tol"], r_tol=case["tol"], max_iter=case["max_iter"])
    AT = torch.load(out_dir / "ATs.pt").numpy()
    RT = torch.load(out_dir / "RTs.pt").numpy()
    Vm = torch.load(out_dir / "Vm.pt").numpy()
    A = sim.A
    if case.get("compact"):
        return compact_fixture(case, sim, AT, RT, Vm, total, iters, wall, step_wall)
    fx = dict(AT=AT, RT=RT, n_total_iter=np.int64(total), iters=np.asarray(iters, dtype=np.int16),
              crow=A.crow_indices().numpy().astype(np.int32), col=A.col_indices().numpy().astype(np.int32),
              wall=np.float64(wall))
    snaps = case.get("snapshots")
    if snaps is None:
        fx["Vm"] = Vm
    else:
        fx["Vm_idx"] = np.asarray(snaps, dtype=np.int32)
        fx["Vm"] = Vm[snaps]
    if case.get("full_matrices"):
        fx["M"] = sim.M.values().numpy()
        fx["K"] = sim.K.values().numpy()
        fx["A"] = sim.A.values().numpy()    # float64 after cg.initialize
        fx["PC"] = sim.pcd.PC.numpy()
    else:
        fx["M_sum"] = np.float64(sim.M.values().double().sum())
        fx["K_abs_sum"] = np.float64(sim.K.values().double().abs().sum())
        fx["A_sum"] = np.float64(sim.A.values().double().sum())
    if traj:
        fx["traj"] = torch.stack(traj).numpy()
    if case.get("phie"):
        fx["Phi_e"] = torch.load(out_dir / "Phi_e.pt").numpy()
    st = states_of(im, case["model"])
    if case.get("keep_states"):
        for k, v in st.items():
            fx["state_" + k] = v
    return fx


def pattern_digest(crow, col):
    """SHA-256 of the CSR pattern as little-endian int32 rowptr then column bytes."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(crow, dtype="<i4").tobytes())
    h.update(np.ascontiguousarray(col, dtype="<i4").tobytes())
    return h.hexdigest()


def time_steps(times, dt):
    """Activation/repolarisation times -> step index n (t_n = n * dt accumulated), -1 where unset."""
    times = np.asarray(times, dtype=np.float64)
    steps = np.where(times < 0, -1, np.rint(times / dt)).astype(np.int64)
    assert steps.max() < 32768
    return steps.astype(np.int16)


def compact_fixture(case, sim, AT, RT, Vm, total, iters, wall, step_wall):
    """Fixture of a full-size case: every node's AT/RT as step indices, Vm on a
    seeded node sample at the listed frames, per-frame statistics over all nodes,
    the pattern digest, matrix sums, per-step iteration counts, reference timing."""
    cp = case["compact"]
    n = AT.shape[0]
    idx = np.sort(np.random.default_rng(cp["seed"]).choice(n, size=min(cp["vm_sample"], n), replace=False))
    frames = np.asarray(cp["vm_frames"], dtype=np.int32)
    Vm64 = Vm.astype(np.float64)
    A = sim.A
    return dict(AT_step=time_steps(AT, case["dt"]), RT_step=time_steps(RT, case["dt"]),
                n_total_iter=np.int64(total), iters=np.asarray(iters, dtype=np.int16),
                pattern_sha256=np.array(pattern_digest(A.crow_indices().numpy(), A.col_indices().numpy())),
                nnz=np.int64(A.col_indices().numel()),
                M_sum=np.float64(sim.M.values().double().sum()),
                K_abs_sum=np.float64(sim.K.values().double().abs().sum()),
                A_sum=np.float64(sim.A.values().double().sum()),
                Vm_nodes=idx.astype(np.int32), Vm_idx=frames, Vm=Vm[frames][:, idx],
                Vm_absmax=np.abs(Vm64).max(axis=1), Vm_mean=Vm64.mean(axis=1), Vm_min=Vm64.min(axis=1),
                wall=np.float64(wall), step_seconds=np.float64(np.sum(step_wall)),
                threads=np.int64(torch.get_num_threads()))


def states_of(im, model):
    if model == "ms":
        names = ["H"]
    elif model == "ttp":
        names = ["CaSR", "CaSS", "Cai", "D", "F", "F2", "FCaSS", "H", "J", "Ki", "M", "Nai", "R", "R_", "S",
                 "Xr1", "Xr2", "Xs"]
    else:
        names = ["Ca_rel", "Ca_up", "Cai", "Ki", "d", "f", "f_Ca", "h", "j", "m", "oa", "oi", "u", "ua", "ui",
                 "v", "w", "xr", "xs"]
    return {n: getattr(im, n).clone().numpy() for n in names}


def run_step_api(md, ionic, case, workdir):
    """Monodomain.step driven step by step (monodomain.py:109-139), as a caller of
    the reference does to change per-node model parameters after initialize():
    assemble, initialize, set the per-node values, then step with the reference's
    own time accumulation; Vm every ``every`` steps and the iteration counts."""
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    mesh_dir = Path(workdir) / case["name"]
    C.write_case_mesh(case, mesh_dir)
    im = make_ionic(ionic, case["model"], case["dt"], dtype, case)
    sim = md.Monodomain(im, T=case["T"], dt=case["dt"], device=torch.device("cpu"), dtype=dtype)
    sim.load_mesh(mesh_dir)
    for cond in case["conductivity"]:
        sim.add_conductivity(**cond)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"], period=s.get("period"), count=s.get("count", 1))
    sim.assemble()
    u = sim.ionic_model.initialize(sim.n_nodes)
    for name, (lo, hi) in case["node_cond"].items():
        setattr(im, name, torch.from_numpy(C.node_values(lo, hi, sim.n_nodes)).to(dtype))
    sim.cg.initialize(x=u, linear_guess=True)
    t = 0.0
    frames, iters = [u.clone()], []
    for k in range(1, int(case["T"] / case["dt"]) + 1):
        t += case["dt"]
        u, it, _, _ = sim.step(u, t, case["tol"], case["tol"], case["max_iter"])
        iters.append(it)
        if k % case["every"] == 0:
            frames.append(u.clone())
    fx = dict(Vm=torch.stack(frames).numpy(), iters=np.asarray(iters, dtype=np.int16))
    for k, v in states_of(im, case["model"]).items():
        fx["state_" + k] = v
    return fx


def run_single_step(ionic, case):
    """One ``differentiate`` on seeded random inputs across the V range."""
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    im = make_ionic(ionic, case["model"], case["dt"], dtype, case)
    V0, st0 = C.random_ionic_inputs(case)
    im.initialize(len(V0))
    for k, v in st0.items():
        setattr(im, k, torch.from_numpy(v).to(dtype))
    dV = im.differentiate(torch.from_numpy(V0).to(dtype))
    fx = dict(V=V0, dV=dV.numpy())
    for k, v in st0.items():
        fx["in_" + k] = v
    for k, v in states_of(im, case["model"]).items():
        fx["out_" + k] = v
    return fx


def run_cell(ionic, case):
    """Single-cell trace: V += dt*dV, plus dt*stim inside the stimulus window."""
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    im = make_ionic(ionic, case["model"], case["dt"], dtype, case)
    V = im.initialize(1)
    dt = case["dt"]
    every = int(round(case["every"] / dt))
    trace = []
    t = 0.0
    for n in range(int(case["T"] / dt)):
        if n % every == 0:
            trace.append(V.item())
        dV = im.differentiate(V)
        V = V + dt * dV
        t += dt
        if case["stim_start"] <= t <= case["stim_start"] + case["stim_dur"]:
            V = V + dt * case["stim"]
    fx = dict(trace=np.asarray(trace), V_end=V.numpy())
    for k, v in states_of(im, case["model"]).items():
        fx["state_" + k] = v
    return fx


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("TORCHCOR_REF"),
                    help="TorchCor checkout to import (default: $TORCHCOR_REF)")
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the TorchCor checkout with --ref or TORCHCOR_REF")
    torch.set_num_threads(a.threads)
    md, ionic = import_reference(a.ref)
    with open(HERE / "cases.json", "w") as f:
        json.dump(C.CASES + C.BIG_CASES, f, indent=1)
    with tempfile.TemporaryDirectory() as work:
        for case in C.CASES + C.BIG_CASES:
            if (a.only and case["name"] not in a.only) or (case.get("big") and not a.only):
                continue
            t0 = time.time()
            kind = case["kind"]
            if kind == "tissue":
                fx = run_tissue(md, ionic, case, work)
            elif kind == "step_api":
                fx = run_step_api(md, ionic, case, work)
            elif kind == "step":
                fx = run_single_step(ionic, case)
            else:
                fx = run_cell(ionic, case)
            np.savez_compressed(HERE / f"{case['name']}.npz", **fx)
            print(case["name"], f"{time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
