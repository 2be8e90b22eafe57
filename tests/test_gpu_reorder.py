"""Node reordering (reverse Cuthill-McKee, Monodomain(..., reorder=True)) is
invisible to the caller: AT/RT, snapshots, the final solution and phi_e come back
in the caller's node numbering and match the reference goldens with the usual
tolerances (AT/RT within one dt, max |dVm| <= 1e-3 max |Vm|, CG iterations within 2 %)."""
import numpy as np
import pytest
import torch

from tests.golden import cases as C
from tests.helpers import case_mesh_dir, device_ionic, golden

pytestmark = pytest.mark.gpu


def _build(case, mesh_dir, device, reorder):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device, reorder=reorder)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"], period=s.get("period"), count=s.get("count", 1))
    return sim


@pytest.mark.parametrize("name", ["ico3_crn_f32", "cube8_ttp_f32", "cube4_ms_period_f32"])
def test_reordered_solve_matches_reference(lib, cuda, tmp_path, name):
    case = C.case(name)
    g = golden(name)
    sim = _build(case, case_mesh_dir(case, tmp_path), cuda, True)
    assert sim.node_order is not None
    sim.solve(case["tol"], case["tol"], case["max_iter"], verbose=False, result_path=tmp_path / "out")
    dt = case["dt"]
    at, rt = sim.activation_time.cpu().numpy(), sim.repolarization_time.cpu().numpy()
    assert np.abs(at - g["AT"]).max() <= dt * 1.001
    assert np.abs(rt - g["RT"]).max() <= dt * 1.001
    vm = sim.solutions.cpu().numpy()
    if "Vm_idx" in g:
        vm = vm[g["Vm_idx"]]
    assert np.abs(vm - g["Vm"]).max() <= 1e-3 * np.abs(g["Vm"]).max()
    assert abs(sim.n_total_iter - int(g["n_total_iter"])) <= max(3, int(g["n_total_iter"]) // 50)
    saved = torch.load(tmp_path / "out" / "ATs.pt").numpy()
    assert np.array_equal(saved, at)
    if "Phi_e" in g:
        phi = sim.phie_recovery(case["tol"], case["tol"], case["max_iter"], Vm=torch.from_numpy(g["Vm"]))
        assert np.abs(phi.cpu().numpy() - g["Phi_e"]).max() <= 1e-4 * np.abs(g["Phi_e"]).max()
