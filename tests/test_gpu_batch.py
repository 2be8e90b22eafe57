"""Batched simulations: every result the same alone and in the mix.

Tolerances as in the single-simulation tests: max |dVm| <= 1e-3 * max |Vm_ref|,
AT/RT within one dt, total CG iterations within 2 %.
"""
import numpy as np
import pytest
import torch

from tests.golden import cases as C
from tests.helpers import case_mesh_dir, device_ionic, golden

pytestmark = pytest.mark.gpu

MIX = ["cube6_ms_f32", "cube8_ttp_f32", "ico3_crn_f32", "cube4_ms_period_f32"]


def build(case, mesh_dir, device):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"], period=s.get("period"), count=s.get("count", 1))
    return sim


def outputs(sim):
    return (sim.activation_time.cpu().numpy(), sim.repolarization_time.cpu().numpy(),
            sim.solutions.cpu().numpy(), sim.n_total_iter)


def assert_close(case, got, ref_at, ref_rt, ref_vm, ref_iters):
    at, rt, vm, iters = got
    dt = case["dt"]
    assert np.abs(at - ref_at).max() <= dt * 1.001
    assert np.abs(rt - ref_rt).max() <= dt * 1.001
    assert np.abs(vm - ref_vm).max() <= 1e-3 * np.abs(ref_vm).max()
    assert abs(iters - ref_iters) <= max(3, ref_iters // 50), (iters, ref_iters)


@pytest.mark.parametrize("variant", [2, 1, 3])
def test_batch_matches_alone_and_reference(lib, cuda, tmp_path, variant):
    """Every batched CG variant (streaming for 2 or 1 blocks per SM, and the one
    staging the ELL streams in shared memory by bulk copies)."""
    from torchcor_b200.simulator import MonodomainBatch
    cases = [C.case(n) for n in MIX]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    alone = []
    for c, d in zip(cases, dirs):
        s = build(c, d, cuda)
        s.solve(c["tol"], c["tol"], c["max_iter"], verbose=False)
        alone.append(outputs(s))
    batch = MonodomainBatch(cuda)
    sims = [batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"]) for c, d in zip(cases, dirs)]
    assert variant in batch.cg_variants()
    batch.set_cg(variant)
    assert batch.cg_config[0] == variant
    batch.run()
    assert not batch.sims
    for c, s, a in zip(cases, sims, alone):
        got = outputs(s)
        assert_close(c, got, *a)
        g = golden(c["name"])
        vm = got[2] if "Vm_idx" not in g else got[2][g["Vm_idx"]]
        assert_close(c, (got[0], got[1], vm, got[3]), g["AT"], g["RT"], g["Vm"], int(g["n_total_iter"]))


def test_batch_join_between_steps(lib, cuda, tmp_path):
    """Simulations that join while others are half way through."""
    from torchcor_b200.simulator import MonodomainBatch
    cases = [C.case(n) for n in ("cube8_ttp_f32", "cube6_ms_f32", "ico3_crn_f32")]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    batch = MonodomainBatch(cuda)
    sims = []
    for k, (c, d) in enumerate(zip(cases, dirs)):
        sims.append(batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"]))
        batch.step(137 * (k + 1))
        for s in batch.finished():
            batch.remove(s)
    batch.run()
    for c, s in zip(cases, sims):
        g = golden(c["name"])
        got = outputs(s)
        vm = got[2] if "Vm_idx" not in g else got[2][g["Vm_idx"]]
        assert_close(c, (got[0], got[1], vm, got[3]), g["AT"], g["RT"], g["Vm"], int(g["n_total_iter"]))


def test_batch_of_one_matches_single_path(lib, cuda, tmp_path):
    from torchcor_b200.simulator import MonodomainBatch
    c = C.case("cfg1_ms_f32")
    d = case_mesh_dir(c, tmp_path)
    single = build(c, d, cuda)
    single.solve(c["tol"], c["tol"], c["max_iter"], verbose=False)
    batch = MonodomainBatch(cuda)
    s = batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"])
    batch.run()
    assert_close(c, outputs(s), *outputs(single))


def test_batch_ionic_tiles_per_block_do_not_change_results(lib, cuda, tmp_path):
    """The batched ionic launch's tiles per block (a tuning knob) only changes which
    block updates which node: every choice gives the same bits."""
    from torchcor_b200 import _lib
    from torchcor_b200.simulator import MonodomainBatch
    cases = [C.case(n) for n in MIX]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    results = {}
    for tpb, bps in ((0, 0), (1, 4), (3, 6), (16, 8), (64, 12), (0, 12)):
        batch = MonodomainBatch(cuda)
        sims = [batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"]) for c, d in zip(cases, dirs)]
        batch.set_ionic(tpb, bps)
        assert (batch.ionic_tiles_per_block, batch.ionic_blocks_per_sm) == (tpb, bps)
        batch.run()
        results[(tpb, bps)] = [outputs(s) for s in sims]
    for tpb, res in results.items():
        for a, b in zip(res, results[(0, 0)]):
            assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3])) and a[3] == b[3], tpb
    batch = MonodomainBatch(cuda)
    with pytest.raises(ValueError):
        batch.set_ionic(65)
    with pytest.raises(ValueError):
        batch.set_ionic(0, 5)
    batch.add(build(cases[0], dirs[0], cuda), cases[0]["tol"], cases[0]["tol"], cases[0]["max_iter"])
    batch.cg_variants()                      # prepares the plan
    assert _lib.load().tcb_batch_set_ionic(C_byref(batch._plan), -1, 0, 0) == _lib.TCB_EINVAL
    assert _lib.load().tcb_batch_set_ionic(C_byref(batch._plan), 0, 7, 0) == _lib.TCB_EINVAL
    assert _lib.load().tcb_batch_set_ionic(C_byref(batch._plan), 0, 12, 1) == _lib.TCB_EINVAL
    assert _lib.load().tcb_batch_set_ionic(C_byref(batch._plan), 0, 0, 2) == _lib.TCB_EINVAL


def test_batch_staged_ionic_matches_alone_and_reference(lib, cuda, tmp_path):
    """The staged batched ionic form (bulk copies of each block's next tile, the
    single-simulation default's division policy) against the simulations alone and
    the reference fixtures, at each register budget; tiles per block do not change
    its bits."""
    from torchcor_b200.simulator import MonodomainBatch
    cases = [C.case(n) for n in MIX]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    alone = []
    for c, d in zip(cases, dirs):
        s = build(c, d, cuda)
        s.solve(c["tol"], c["tol"], c["max_iter"], verbose=False)
        alone.append(outputs(s))
    bits = {}
    for tpb, bps in ((0, 4), (0, 6), (0, 8), (2, 6)):
        batch = MonodomainBatch(cuda)
        sims = [batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"]) for c, d in zip(cases, dirs)]
        assert batch.ionic_stage_ok()
        batch.set_ionic(tpb, bps, staged=True)
        assert batch.ionic_staged == 1
        batch.run()
        got_all = [outputs(s) for s in sims]
        for c, got, a in zip(cases, got_all, alone):
            assert_close(c, got, *a)
            g = golden(c["name"])
            vm = got[2] if "Vm_idx" not in g else got[2][g["Vm_idx"]]
            assert_close(c, (got[0], got[1], vm, got[3]), g["AT"], g["RT"], g["Vm"], int(g["n_total_iter"]))
        bits.setdefault(bps, got_all)
        if (tpb, bps) == (2, 6):
            for a, b in zip(got_all, bits[6]):
                assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3])) and a[3] == b[3]
    batch = MonodomainBatch(cuda)
    with pytest.raises(ValueError):
        batch.set_ionic(0, 12, staged=True)       # no 12-block budget for the staged form


def C_byref(x):
    import ctypes
    return ctypes.byref(x)


def test_batch_autotune_choice_is_cached_and_results_hold(lib, cuda, tmp_path):
    """The tuner times real steps of the batch with each CG variant, keeps the
    fastest, caches it, and the simulations still match the reference."""
    from torchcor_b200.simulator import MonodomainBatch
    from torchcor_b200.tune import BATCH_IONIC_BPS, BATCH_IONIC_TPB, CG_VARIANTS, TuneCache, tune_batch
    cases = [C.case(n) for n in ("cube6_ms_f32", "cube8_ttp_f32")]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    cache = TuneCache(tmp_path / "tune.json")
    batch = MonodomainBatch(cuda)
    sims = [batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"]) for c, d in zip(cases, dirs)]
    choice, times = tune_batch(batch, steps=3, cache=cache)
    assert choice in CG_VARIANTS and set(times) == set(batch.cg_variants())
    assert batch.cg_config[0] == choice
    entry = next(iter(cache.load().values()))
    assert len(cache.load()) == 1 and entry["ionic_tiles_per_block"] in BATCH_IONIC_TPB
    assert batch.ionic_tiles_per_block == entry["ionic_tiles_per_block"]
    assert set(entry["ionic_ms_per_step"]) == {str(t) for t in BATCH_IONIC_TPB}
    assert entry["ionic_blocks_per_sm"] in BATCH_IONIC_BPS
    assert batch.ionic_blocks_per_sm == entry["ionic_blocks_per_sm"]
    assert batch.ionic_staged == entry["ionic_staged"]
    assert set(entry["ionic_staged_ms_per_step"]) == {"4", "6", "8"}
    batch.set_ionic(0, 0, 0)
    again, t2 = tune_batch(batch, steps=3, cache=cache)
    assert again == choice and t2 is None          # served from the cache
    assert batch.ionic_tiles_per_block == entry["ionic_tiles_per_block"]
    assert batch.ionic_staged == entry["ionic_staged"]
    batch.run()
    for c, s in zip(cases, sims):
        g = golden(c["name"])
        got = outputs(s)
        vm = got[2] if "Vm_idx" not in g else got[2][g["Vm_idx"]]
        assert_close(c, (got[0], got[1], vm, got[3]), g["AT"], g["RT"], g["Vm"], int(g["n_total_iter"]))


def test_batch_with_mixed_code_paths(lib, cuda, tmp_path):
    """A batch whose simulations do not share one (int16 columns, A rebuilt,
    linear guess) combination runs the kernel that picks the path per slice;
    a uniform batch runs the specialised kernel.  Results as alone."""
    from torchcor_b200.simulator import MonodomainBatch
    cases = [C.case(n) for n in ("cube6_ms_f32", "cube8_ttp_f32")]
    dirs = [case_mesh_dir(c, tmp_path) for c in cases]
    alone = []
    for k, (c, d) in enumerate(zip(cases, dirs)):
        s = build(c, d, cuda)
        s.solve(c["tol"], c["tol"], c["max_iter"], verbose=False, linear_guess=k == 0)
        alone.append(outputs(s))
    batch = MonodomainBatch(cuda)
    sims = [batch.add(build(c, d, cuda), c["tol"], c["tol"], c["max_iter"], linear_guess=k == 0)
            for k, (c, d) in enumerate(zip(cases, dirs))]
    batch.step(1)
    assert batch._plan.cg_flags == -1
    batch.run()
    for c, s, a in zip(cases, sims, alone):
        assert_close(c, outputs(s), *a)
    uniform = MonodomainBatch(cuda)
    uniform.add(build(cases[0], dirs[0], cuda), 1e-5, 1e-5, 100)
    uniform.step(1)
    assert uniform._plan.cg_flags == 7
