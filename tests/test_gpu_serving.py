"""Serving loop on the GPU: requests that arrive while others run give the
results of the same simulations run alone (final Vm within 1e-3 of its maximum
magnitude, AT/RT within one dt, total CG iterations within 2 %)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_requests_match_alone(lib, cuda):
    from torchcor_b200 import serving
    reqs = [serving.Request(0, 0.0, "cube", 6, "ms", 30.0),
            serving.Request(1, 0.02, "ico", 3, "crn", 20.0),
            serving.Request(2, 0.05, "cube", 5, "ttp", 25.0),
            serving.Request(3, 0.06, "ico", 4, "ms", 15.0)]
    server = serving.Server(cuda, round_steps=37)
    summary = server.run(reqs)
    assert summary["requests"] == 4 and summary["latency_p99_s"] >= summary["latency_p50_s"] > 0
    for r in reqs:
        alone = serving.build_sim(r, cuda)
        alone.solve(r.a_tol, r.r_tol, r.max_iter, verbose=False, snapshot_interval=r.T)
        at, rt = alone.activation_time.cpu().numpy(), alone.repolarization_time.cpu().numpy()
        assert np.abs(r.result["AT"].numpy() - at).max() <= r.dt * 1.001
        assert np.abs(r.result["RT"].numpy() - rt).max() <= r.dt * 1.001
        vm = alone.current_solution().cpu().numpy()
        assert np.abs(r.result["Vm"].numpy() - vm).max() <= 1e-3 * np.abs(vm).max()
        assert abs(r.n_total_iter - alone.n_total_iter) <= max(3, alone.n_total_iter // 50)


@pytest.mark.parametrize("mesh,size", [("cube", 79), ("ico", 8)])
@pytest.mark.parametrize("model", ["ms", "ttp", "crn"])
def test_admission_estimate_covers_device_memory(lib, cuda, mesh, size, model):
    """The server admits requests by serving.footprint_bytes; a request of the large
    end of the mix (512,000-node cube, 655,362-node icosphere) must not hold more
    device memory than that estimate once built and added to a batch."""
    import gc

    import torch
    from torchcor_b200 import serving
    from torchcor_b200.simulator import MonodomainBatch
    req = serving.Request(0, 0.0, mesh, size, model, 50.0)
    batch = MonodomainBatch(cuda)
    gc.collect()                       # earlier tests' tensors are released before the baseline
    torch.cuda.synchronize(cuda)
    base = torch.cuda.memory_allocated(cuda)
    torch.cuda.reset_peak_memory_stats(cuda)
    sim = serving.build_sim(req, cuda)
    sim.prepare(req.a_tol, req.r_tol, req.max_iter, snapshot_interval=req.T)
    batch.add(sim, req.a_tol, req.r_tol, req.max_iter, snapshot_interval=req.T)
    batch.step(1)
    torch.cuda.synchronize(cuda)
    held = torch.cuda.memory_allocated(cuda) - base
    peak = torch.cuda.max_memory_allocated(cuda) - base
    est = serving.footprint_bytes(req)
    print(f"{mesh}{size} {model}: nodes {req.n_nodes}, held {held / 2**20:.0f} MiB, "
          f"build peak {peak / 2**20:.0f} MiB, estimate {est / 2**20:.0f} MiB")
    assert held <= est, (held, est)
