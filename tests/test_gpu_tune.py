"""Launch-shape tuning of the single-simulation kernels on a GPU.

Every instance of the fused ionic kernel (nodes per thread, register budget,
division policy) must compute the same step as the default instance up to the
few-ulp differences of the division policy; the tuner must set its choice in
the simulation, record it in the cache and leave the simulation untouched.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.golden import cases as CS
from tests.helpers import case_mesh_dir, device_ionic

pytestmark = pytest.mark.gpu


def _prepared(case, mesh_dir, device):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"])
    sim.prepare(case["tol"], case["tol"], case["max_iter"])
    return sim


@pytest.mark.parametrize("name", ["cube6_ms_f32", "cube8_ttp_f32", "ico3_crn_f32"])
def test_ionic_instances_agree(lib, cuda, tmp_path, name):
    from torchcor_b200 import _lib, tune
    case = CS.case(name)
    sim = _prepared(case, case_mesh_dir(case, tmp_path), cuda)
    stream = torch.cuda.current_stream(cuda)
    _lib.check(lib.tcb_mono_run(C.byref(sim._sim["struct"]), 1, 31, stream.cuda_stream))   # into the upstroke
    sim._sim["next_step"] = 31
    before = sim.ionic_model.state.clone()
    scratch = tune.ScratchSim(sim)
    shapes = _lib.ionic_variants(sim.ionic_model.model_id)
    assert len(shapes) >= 3
    ref = None
    for k in range(1, len(shapes) + 1):
        scratch.struct.ionic_variant = k
        tune.time_steps(scratch, 31, 20, stream)
        out = (scratch.buf["state"][:, : sim.n_nodes].clone(), scratch.buf["x"][:, : sim.n_nodes].clone(),
               scratch.buf["at_rt"][:, : sim.n_nodes].clone())
        if ref is None:
            ref = out
            continue
        for got, want in zip(out[:2], ref[:2]):
            err = (got - want).abs().max().item() / max(want.abs().max().item(), 1e-30)
            assert err <= 5e-4, (k, shapes[k - 1], err)
        assert (out[2] - ref[2]).abs().max().item() <= case["dt"] * 1.001
    assert torch.equal(sim.ionic_model.state, before)        # trials ran on the copy


def test_tuner_sets_and_caches_its_choice(lib, cuda, tmp_path):
    from torchcor_b200 import _lib, tune
    case = CS.case("cube8_ttp_f32")
    sim = _prepared(case, case_mesh_dir(case, tmp_path), cuda)
    cache = tune.TuneCache(tmp_path / "tune.json")
    x0 = sim._sim["x"].clone()
    got = tune.tune_single(sim, steps=3, cache=cache)
    assert got["measured"] and got["ionic_variant"] >= 1
    st = sim._sim["struct"]
    assert st.ionic_variant == got["ionic_variant"] and st.cg_per_sm == got["cg_per_sm"]
    assert len(got["ionic_ms"]) == len(_lib.ionic_variants(_lib.MODEL_TTP))
    assert torch.equal(sim._sim["x"], x0) and sim._sim["next_step"] == 1
    again = tune.tune_single(sim, steps=3, cache=cache)
    assert again.get("cached") and again["ionic_variant"] == got["ionic_variant"]
    total = sim.solve(case["tol"], case["tol"], case["max_iter"], verbose=False, autotune=False)
    assert total > 0


@pytest.mark.parametrize("name", ["cube6_ms_f32", "cube8_ttp_f32", "ico3_crn_f32"])
def test_fused_step_equals_two_launches(lib, cuda, tmp_path, name):
    """The step as one launch (ionic update inside the resident CG kernel) gives the
    two-launch step's values bit for bit: same sums in the same order."""
    from torchcor_b200 import _lib
    case = CS.case(name)
    d = case_mesh_dir(case, tmp_path)
    sims = [_prepared(case, d, cuda) for _ in range(2)]
    for sim, fused in zip(sims, (0, 1)):
        sim.set_launch(ionic_variant=1, cg_per_sm=0, fused_step=fused)
    st = [s._sim["struct"] for s in sims]
    assert lib.tcb_mono_cg_kernel(C.byref(st[0])) == 1 and lib.tcb_mono_cg_kernel(C.byref(st[1])) == 2
    nt = sims[0].nt
    for sim, m in zip(sims, st):
        _lib.check(lib.tcb_mono_run(C.byref(m), 1, nt + 1, _lib.stream_ptr()))
        _lib.check(lib.tcb_mono_check(C.byref(m), _lib.stream_ptr()))
    a, b = (s._sim for s in sims)
    assert torch.equal(a["step_iters"], b["step_iters"])
    # instance 1 of each model and its fused step share the division policy
    for key in ("x", "at_rt"):
        assert torch.equal(a[key], b[key]), key
    assert torch.equal(sims[0].ionic_model.state, sims[1].ionic_model.state)
