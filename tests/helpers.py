"""Helpers shared by the tests: golden fixtures and case construction."""
from __future__ import annotations

import tempfile
from pathlib import Path

import numpy as np
import torch

from tests.golden import cases as C

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


def oracle_ionic(case):
    from oracle import port as P
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    if case["model"] == "ms":
        return P.ModifiedMS2v(case["dt"], dtype)
    if case["model"] == "ttp":
        return P.TenTusscherPanfilov(case.get("cell_type", "ENDO"), case["dt"], dtype)
    return P.CourtemancheRamirezNattel(case["dt"], dtype)


def device_ionic(case, device):
    from torchcor_b200 import ionic
    if case["model"] == "ms":
        return ionic.ModifiedMS2v(case["dt"], device=device)
    if case["model"] == "ttp":
        return ionic.TenTusscherPanfilov(case.get("cell_type", "ENDO"), case["dt"], device=device)
    return ionic.CourtemancheRamirezNattel(case["dt"], device=device)


def run_oracle_tissue(case, mesh_dir, **kw):
    from oracle import port as P
    dtype = torch.float64 if case["dtype"] == "f64" else torch.float32
    sim = P.Monodomain(oracle_ionic(case), case["T"], case["dt"], dtype)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(Path(mesh_dir) / s["file"]), s["start"], s["duration"], s["intensity"],
                         s.get("period"), s.get("count", 1))
    return sim, sim.solve(case["tol"], case["tol"], case["max_iter"], **kw)


def run_device_tissue(case, mesh_dir, device, result_dir=None, launch=None):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(Path(mesh_dir) / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"], period=s.get("period"), count=s.get("count", 1))
    total = sim.solve(a_tol=case["tol"], r_tol=case["tol"], max_iter=case["max_iter"], calculate_AT_RT=True,
                      linear_guess=True, snapshot_interval=1, verbose=False, result_path=result_dir, launch=launch)
    return sim, total


def case_mesh_dir(case, root):
    d = Path(root) / case["name"]
    C.write_case_mesh(case, d)
    return d


def record_parity(case_name, reference, **metrics):
    """Append one measured-error record (JSON line) to $TCB_PARITY_REPORT, if set."""
    import json
    import os
    path = os.environ.get("TCB_PARITY_REPORT")
    if not path:
        return
    rec = {"case": case_name, "reference": reference}
    rec.update({k: (float(v) if isinstance(v, (np.floating, float)) else int(v) if isinstance(v, (np.integer, int))
                    else v) for k, v in metrics.items()})
    with open(path, "a") as f:
        f.write(json.dumps(rec) + "\n")
