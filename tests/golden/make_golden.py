"""Generate the golden fixtures in this directory by running the TorchCor
reference itself (pure Python/PyTorch, CPU).

Run from the repository root, where the reference checkout is mounted:

    python tests/golden/make_golden.py [--ref /root/reference] [--only name ...]

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
import json
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

    def step(u, t, a_tol, r_tol, max_iter, verbose=False):
        out = orig_step(u, t, a_tol, r_tol, max_iter, verbose)
        iters.append(out[1])
        if len(traj) < case.get("keep_steps", 0):
            traj.append(out[0].clone())
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
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    torch.set_num_threads(a.threads)
    md, ionic = import_reference(a.ref)
    with open(HERE / "cases.json", "w") as f:
        json.dump(C.CASES, f, indent=1)
    with tempfile.TemporaryDirectory() as work:
        for case in C.CASES:
            if a.only and case["name"] not in a.only:
                continue
            t0 = time.time()
            kind = case["kind"]
            if kind == "tissue":
                fx = run_tissue(md, ionic, case, work)
            elif kind == "step":
                fx = run_single_step(ionic, case)
            else:
                fx = run_cell(ionic, case)
            np.savez_compressed(HERE / f"{case['name']}.npz", **fx)
            print(case["name"], f"{time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
