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
def test_fused_step_matches_two_launches(lib, cuda, tmp_path, name):
    """The step as one launch (ionic update inside the resident CG kernel) against
    the two-launch step, from the same state (step 31, in the upstroke) over 20
    steps: the same sums in the same order, so the only differences are the
    multiply-add contractions the compiler picks for the inlined ionic update in
    each kernel (last bits of b'): solutions within 1e-5 of their range, the same
    CG iteration counts.  Ionic states within 1e-5 too, except where a gate's
    update switches at a voltage threshold (Mitchell-Schaeffer's h at u_gate): a
    node sitting on the threshold may take the other branch, so the states are
    held to 1e-2 there."""
    from torchcor_b200 import _lib, tune
    case = CS.case(name)
    sim = _prepared(case, case_mesh_dir(case, tmp_path), cuda)
    stream = torch.cuda.current_stream(cuda)
    _lib.check(lib.tcb_mono_run(C.byref(sim._sim["struct"]), 1, 31, stream.cuda_stream))
    sim._sim["next_step"] = 31
    scratch = tune.ScratchSim(sim)
    # the two-launch step with the first one-node instance of the fused kernel's
    # division policy (IEEE for MS and TTP, hardware for CRN)
    fast = 1 if sim.ionic_model.model_id == _lib.MODEL_CRN else 0
    k = 1 + next(i for i, sh in enumerate(_lib.ionic_variants(sim.ionic_model.model_id))
                 if sh[0] == 1 and sh[2] == fast and sh[3] == 0)
    out = []
    for fused in (0, 1):
        m = scratch.struct
        m.ionic_variant, m.cg_per_sm, m.fused_step = k if not fused else 1, 0, fused
        assert lib.tcb_mono_cg_kernel(C.byref(m)) == (2 if fused else 1)
        tune.time_steps(scratch, 31, 20, stream)
        out.append({k: scratch.buf[k].clone() for k in ("x", "at_rt", "step_iters", "state")})
    a, b = out
    assert torch.equal(a["step_iters"], b["step_iters"])
    for k, tol in (("x", 1e-5), ("state", 1e-2 if name.startswith("cube6_ms") else 1e-5)):
        err = (a[k] - b[k]).abs().max().item() / a[k].abs().max().item()
        assert err <= tol, (k, err)
    assert (a["at_rt"] - b["at_rt"]).abs().max().item() <= case["dt"] * 1.001
