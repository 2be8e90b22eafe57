"""tcb_mono_run_noalloc: the time loop for callers that cannot allocate device
memory at the call site (a host application owning the device memory pool, a
latency-critical caller that cannot take cudaMalloc's implicit
synchronisation).  Its CG scratch lives in a static device array of the
library, so the caller passes no scratch buffers.

Checked through the C ABI against tcb_mono_run on the same simulation, on two
calls in a row, with each CG kernel: the results agree bit for bit.  This file is
collected last, so a stop-at-first-failure run has already run every other
test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.golden import cases as CS
from tests.helpers import case_mesh_dir, device_ionic

pytestmark = pytest.mark.gpu


def prepared(case, mesh_dir, device):
    from torchcor_b200.simulator import Monodomain
    sim = Monodomain(device_ionic(case, device), T=case["T"], dt=case["dt"], device=device)
    sim.load_mesh(mesh_dir)
    for c in case["conductivity"]:
        sim.add_conductivity(**c)
    for s in case["stimuli"]:
        sim.add_stimulus(str(mesh_dir / s["file"]), start=s["start"], duration=s["duration"],
                         intensity=s["intensity"])
    sim.assemble()
    sim._setup(case["tol"], case["tol"], case["max_iter"], True, True, 1, False)
    return sim


@pytest.mark.parametrize("kernel", ["resident", "streaming"])
def test_noalloc_matches_allocating_entry_point(lib, cuda, tmp_path, monkeypatch, kernel):
    """Both CG kernels (the one keeping rows in shared memory and the streaming
    one) use the static scratch; the kernels are deterministic (fixed-order
    reductions, no float atomics), so the two entry points agree bit for bit."""
    from torchcor_b200._lib import check, stream_ptr
    if kernel == "streaming":
        monkeypatch.setenv("TCB_CG_KERNEL", "streaming")
    case = CS.case("cube6_ms_f32")
    d = case_mesh_dir(case, tmp_path)
    ref = prepared(case, d, cuda)
    new = prepared(case, d, cuda)
    st = new._sim["struct"]
    st.scratch = None          # the no-allocation entry point must not need these
    st.barrier = None
    n = ref.nt // 2
    for call, (a, b) in enumerate([(1, n + 1), (n + 1, ref.nt + 1)]):
        check(lib.tcb_mono_run(C.byref(ref._sim["struct"]), a, b, stream_ptr()))
        check(lib.tcb_mono_run_noalloc(C.byref(st), a, b, stream_ptr()))
        check(lib.tcb_mono_check(C.byref(ref._sim["struct"]), stream_ptr()))
        check(lib.tcb_mono_check(C.byref(st), stream_ptr()))
        ref._sim["next_step"] = new._sim["next_step"] = b
        u_ref = ref.current_solution().cpu().numpy()
        u_new = new.current_solution().cpu().numpy()
        assert np.array_equal(u_new, u_ref), call
        assert np.array_equal(new._sim["step_iters"][a:b].cpu().numpy(), ref._sim["step_iters"][a:b].cpu().numpy())
        at_ref = ref._sim["at"].cpu().numpy()
        at_new = new._sim["at"].cpu().numpy()
        assert np.array_equal(at_new, at_ref), call
    assert int(new._sim["counter"][0].item()) == ref.nt + 1
