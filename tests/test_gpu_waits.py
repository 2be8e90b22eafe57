"""Failure detection of the bounded device waits, without a GPU fault.

Every device-side wait (the grid barriers of the persistent CG kernels, the
mbarriers of the batched kernels' bulk copies) gives up after a time limit,
records TCB_ETIMEOUT in the simulation's error word and returns, so a lost
block or copy can never hang the GPU.  The internal test variable
TCB_TEST_WAIT_STALL makes such a wait run out on purpose (limit 10 ms):
"grid" makes every grid barrier wait for one arrival more than the grid has,
"copy" leaves the first bulk copies of a staged batched kernel (the first warp
of the batched CG kernel, the first block of the staged batched ionic kernel)
unissued while their mbarrier still expects the bytes.  The tests check the reported
status and that the next normal run on the same GPU is correct.
"""
import ctypes as C

import numpy as np
import pytest

from tests.golden import cases as CS
from tests.helpers import case_mesh_dir, device_ionic, golden

pytestmark = pytest.mark.gpu


def _sim(case, mesh_dir, device):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"])
    return sim


def _clean_solve_matches_reference(case, mesh_dir, device):
    g = golden(case["name"])
    sim = _sim(case, mesh_dir, device)
    total = sim.solve(case["tol"], case["tol"], case["max_iter"], verbose=False)
    at = sim.activation_time.cpu().numpy()
    assert np.abs(at - g["AT"]).max() <= case["dt"] * 1.001
    assert abs(total - int(g["n_total_iter"])) <= max(3, int(g["n_total_iter"]) // 50)


@pytest.mark.parametrize("kernel", ["resident", "streaming"])
def test_grid_barrier_timeout_is_reported(lib, cuda, tmp_path, monkeypatch, kernel):
    from torchcor_b200 import _lib
    case = CS.case("cube6_ms_f32")
    d = case_mesh_dir(case, tmp_path)
    if kernel == "streaming":
        monkeypatch.setenv("TCB_CG_KERNEL", "streaming")
    sim = _sim(case, d, cuda)
    sim.prepare(case["tol"], case["tol"], case["max_iter"])
    st = sim._sim["struct"]
    assert lib.tcb_mono_cg_kernel(C.byref(st)) == (1 if kernel == "resident" else 0)
    monkeypatch.setenv("TCB_TEST_WAIT_STALL", "grid")
    _lib.check(lib.tcb_mono_run(C.byref(st), 1, 4, _lib.stream_ptr()))   # the launches themselves succeed
    assert lib.tcb_mono_check(C.byref(st), _lib.stream_ptr()) == _lib.TCB_ETIMEOUT
    assert int(sim._sim["counter"][1].item()) == _lib.TCB_ETIMEOUT       # the device error word
    monkeypatch.delenv("TCB_TEST_WAIT_STALL")
    # the context is usable: a fresh solve on the same GPU is correct
    _clean_solve_matches_reference(case, d, cuda)


def test_bulk_copy_wait_timeout_is_reported(lib, cuda, tmp_path, monkeypatch):
    from torchcor_b200 import _lib
    from torchcor_b200.simulator import MonodomainBatch
    case = CS.case("cube6_ms_f32")
    d = case_mesh_dir(case, tmp_path)
    monkeypatch.setenv("TCB_TEST_WAIT_STALL", "copy")     # read when the batch plan is prepared
    batch = MonodomainBatch(cuda)
    batch.add(_sim(case, d, cuda), case["tol"], case["tol"], case["max_iter"])
    assert 3 in batch.cg_variants()
    batch.set_cg(3)                                        # ELL streams staged by bulk copies
    assert batch.cg_config[0] == 3
    batch.step(2)
    with pytest.raises(_lib.TcbError) as e:
        batch.check()
    assert e.value.status == _lib.TCB_ETIMEOUT
    monkeypatch.delenv("TCB_TEST_WAIT_STALL")
    _clean_solve_matches_reference(case, d, cuda)


def test_staged_batched_ionic_copy_wait_timeout_is_reported(lib, cuda, tmp_path, monkeypatch):
    """The staged batched ionic kernel: block 0's first tile copies are not made while
    its mbarrier expects the bytes; the bounded wait runs out and is reported."""
    from torchcor_b200 import _lib
    from torchcor_b200.simulator import MonodomainBatch
    case = CS.case("cube8_ttp_f32")
    d = case_mesh_dir(case, tmp_path)
    monkeypatch.setenv("TCB_TEST_WAIT_STALL", "copy")     # read when the batch plan is prepared
    batch = MonodomainBatch(cuda)
    batch.add(_sim(case, d, cuda), case["tol"], case["tol"], case["max_iter"])
    batch.set_cg(2)                                        # streaming CG: no copies of its own
    batch.set_ionic(0, 6, staged=True)
    assert batch.ionic_staged == 1
    batch.step(2)
    with pytest.raises(_lib.TcbError) as e:
        batch.check()
    assert e.value.status == _lib.TCB_ETIMEOUT
    monkeypatch.delenv("TCB_TEST_WAIT_STALL")
    _clean_solve_matches_reference(case, d, cuda)
