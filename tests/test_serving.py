"""Serving workload generator and footprint estimate (CPU)."""
import numpy as np

from torchcor_b200 import serving


def test_requests_seeded_and_shaped():
    a = serving.generate_requests(count=200, seed=7)
    b = serving.generate_requests(count=200, seed=7)
    assert [(r.mesh, r.size, r.model, r.T, r.arrival_s) for r in a] == \
           [(r.mesh, r.size, r.model, r.T, r.arrival_s) for r in b]
    arr = np.array([r.arrival_s for r in a])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert all(50.0 <= r.T <= 300.0 for r in a)
    assert {r.model for r in a} == set(serving.MODELS)
    assert {r.mesh for r in a} == {"cube", "ico"}
    for r in a:
        if r.mesh == "cube":
            assert 10_000 * 0.5 < r.n_nodes < 500_000 * 1.1
        else:
            assert r.size in serving.ICO_LEVEL_NODES


def test_offered_load_matches_rate():
    reqs = serving.generate_requests(count=2000, seed=3, capacity=4e9, load=0.8)
    work = sum(r.n_nodes * r.nt for r in reqs)
    span = reqs[-1].arrival_s
    assert 0.7 < work / span / 4e9 < 0.9   # Poisson: offered load near 0.8 of the capacity


def test_footprint_grows_with_size_and_model():
    small = serving.Request(0, 0.0, "cube", 20, "ms", 100.0)
    big = serving.Request(0, 0.0, "cube", 40, "ms", 100.0)
    ttp = serving.Request(0, 0.0, "cube", 20, "ttp", 100.0)
    assert 0 < serving.footprint_bytes(small) < serving.footprint_bytes(big)
    assert serving.footprint_bytes(small) < serving.footprint_bytes(ttp)
