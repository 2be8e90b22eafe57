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
