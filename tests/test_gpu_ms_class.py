"""The ``MitchellSchaeffer`` drop-in class in both constructor forms.

The reference's ``Monodomain`` runs the dimensional two-variable model
(torchcor/ionic/ModifiedMS2v.py:36-44); the class named ``MitchellSchaeffer``
here is that model and accepts the reference's own constructor form
``MitchellSchaeffer(device, dtype)`` (torchcor/ionic/MitchellSchaeffer.py:6-23,
ionic/base.py:30: no dt, the simulator supplies it) as well as
``MitchellSchaeffer(dt, device=..., dtype=...)``.  Both run the 20^3 cube
(9,261 nodes, T = 50 ms) and must match the reference's fixture of that case.
"""
import numpy as np
import pytest
import torch

from tests.golden import cases as C
from tests.helpers import case_mesh_dir, golden

pytestmark = pytest.mark.gpu


def _run(model, case, mesh_dir, out):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(model, T=case["T"], dt=case["dt"], device=model.device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"])
    total = sim.solve(a_tol=case["tol"], r_tol=case["tol"], max_iter=case["max_iter"], calculate_AT_RT=True,
                      linear_guess=True, snapshot_interval=1, verbose=False, result_path=str(out))
    return sim, total


@pytest.mark.parametrize("form", ["reference", "with_dt"])
def test_mitchell_schaeffer_class_runs_cfg1(lib, cuda, form, tmp_path):
    from torchcor_b200.ionic import MitchellSchaeffer
    case = C.case("cfg1_ms_f32")
    g = golden("cfg1_ms_f32")
    if form == "reference":
        model = MitchellSchaeffer(cuda, torch.float32)      # dt comes from Monodomain
        assert model.dt is None
    else:
        model = MitchellSchaeffer(case["dt"], device=cuda, dtype=torch.float32)
    out = tmp_path / "out"
    sim, total = _run(model, case, case_mesh_dir(case, tmp_path), out)
    assert model.dt == case["dt"] and model.name == "MitchellSchaeffer"
    AT = torch.load(out / "ATs.pt").numpy()
    Vm = torch.load(out / "Vm.pt").numpy()[g["Vm_idx"]]
    assert (AT > 0).all()                                    # the whole cube activates
    assert np.abs(AT - g["AT"]).max() <= case["dt"] * 1.001
    assert np.abs(Vm - g["Vm"]).max() <= 1e-3 * np.abs(g["Vm"]).max()
    ref_total = int(g["n_total_iter"])
    assert abs(total - ref_total) <= max(3, ref_total // 50)
