"""Streamed snapshot output (solve(..., snapshot_ring=R)): only R frames on the
device, every frame copied to pinned host memory as soon as it is written; the
frames, AT/RT and Vm.pt must be bit-identical to the default (every frame kept on
the device), for rings smaller than the number of frames, one frame per step, and
with node reordering.  The default writes Vm.pt while the steps run
(resultio.FrameWriter): its file must be torch.save's file of the frames."""
import zipfile

import numpy as np
import pytest
import torch

from tests.golden import cases as C
from tests.helpers import case_mesh_dir
from tests.test_gpu_reorder import _build

pytestmark = pytest.mark.gpu


def _run(case, d, cuda, tmp, ring, interval, reorder=False, graph_steps=100):
    sim = _build(case, d, cuda, reorder)
    sim.solve(case["tol"], case["tol"], case["max_iter"], verbose=False, snapshot_interval=interval,
              result_path=tmp, snapshot_ring=ring, graph_steps=graph_steps)
    return sim


@pytest.mark.parametrize("name,interval,ring,reorder", [
    ("cube6_ms_f32", 1.0, 2, False),      # frames every 100 steps, ring of 2
    ("cube4_ms_period_f32", 0.01, 3, False),   # a frame every step
    ("ico3_crn_f32", 2.0, 1, True),      # ring of one row, reordered nodes
])
def test_streamed_snapshots_equal_device_snapshots(lib, cuda, tmp_path, name, interval, ring, reorder):
    case = C.case(name)
    d = case_mesh_dir(case, tmp_path)
    ref = _run(case, d, cuda, tmp_path / "a", None, interval, reorder)
    got = _run(case, d, cuda, tmp_path / "b", ring, interval, reorder)
    assert got.solutions.device.type == "cpu"
    assert got.solutions.is_pinned() or reorder      # reordering gathers into a new host tensor
    assert got.solutions.shape[0] > ring
    assert torch.equal(got.solutions, ref.solutions.cpu())
    assert torch.equal(got.activation_time.cpu(), ref.activation_time.cpu())
    assert torch.equal(got.repolarization_time.cpu(), ref.repolarization_time.cpu())
    assert torch.equal(torch.load(tmp_path / "b" / "Vm.pt"), torch.load(tmp_path / "a" / "Vm.pt"))


@pytest.mark.parametrize("name,interval,ring,graph_steps", [
    ("cube6_ms_f32", 1.0, None, 7),       # whole loop in one chunk: 1 plain step, 7-step replays, a plain tail
    ("cube6_ms_f32", 1.0, 2, 7),          # streamed snapshots: replays inside every 100-step frame
    ("ico3_crn_f32", 2.0, None, 100),
])
def test_graph_replay_equals_plain_launches(lib, cuda, tmp_path, name, interval, ring, graph_steps):
    case = C.case(name)
    d = case_mesh_dir(case, tmp_path)
    ref = _run(case, d, cuda, tmp_path / "a", ring, interval, graph_steps=0)
    got = _run(case, d, cuda, tmp_path / "b", ring, interval, graph_steps=graph_steps)
    assert got._sim.get("graph") is not None and ref._sim.get("graph") is None
    assert torch.equal(got.solutions.cpu(), ref.solutions.cpu())
    assert torch.equal(got.activation_time.cpu(), ref.activation_time.cpu())
    assert torch.equal(got.repolarization_time.cpu(), ref.repolarization_time.cpu())
    assert torch.equal(got._sim["step_iters"].cpu(), ref._sim["step_iters"].cpu())


def test_frame_writer_follows_the_compute_stream(cuda, tmp_path):
    from torchcor_b200.simulator.resultio import FrameWriter
    g = torch.Generator(device=cuda).manual_seed(3)
    src = torch.randn(9, 40_000, device=cuda, generator=g)
    frames = torch.zeros_like(src)
    w = FrameWriter(tmp_path / "Vm.pt", frames)
    cur = torch.cuda.current_stream(cuda)
    for k in range(src.shape[0] - 1):
        torch.cuda._sleep(200_000)              # the frame is produced well after the mark is posted
        frames[k].copy_(src[k] * 2.0)
        ev = torch.cuda.Event()
        ev.record(cur)
        w.produced(k + 1, ev)
    frames[-1].copy_(src[-1] * 2.0)
    ev = torch.cuda.Event()
    ev.record(cur)
    w.finish(ev)
    assert torch.equal(torch.load(tmp_path / "Vm.pt"), (src * 2.0).cpu())
    with zipfile.ZipFile(tmp_path / "Vm.pt") as z:
        assert z.testzip() is None


def test_frame_writer_abort_ends_the_thread(cuda, tmp_path):
    from torchcor_b200.simulator.resultio import FrameWriter
    frames = torch.zeros(4, 1000, device=cuda)
    w = FrameWriter(tmp_path / "Vm.pt", frames)
    ev = torch.cuda.Event()
    ev.record()
    w.produced(2, ev)
    w.abort()
    assert not w._thread.is_alive()
    with pytest.raises(RuntimeError):
        w.finish(ev)


def test_solve_streams_vm_file_equal_to_saved_frames(lib, cuda, tmp_path):
    case = C.case("cube6_ms_f32")
    d = case_mesh_dir(case, tmp_path)
    sim = _run(case, d, cuda, tmp_path / "a", None, 1.0)
    with zipfile.ZipFile(tmp_path / "a" / "Vm.pt") as z:
        assert z.testzip() is None
    assert torch.equal(torch.load(tmp_path / "a" / "Vm.pt"), sim.solutions.cpu())
