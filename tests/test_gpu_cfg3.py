"""The CRN icosphere at full size: a level-7 icosphere (163,842 nodes, 327,680
triangles, radius 25 mm), seeded random tangent fibres, il/it = 0.4/0.1, the cap
z > 24.5 mm stimulated for 2 ms at intensity 50, dt 0.02 ms.  The float32 device
path (float64 CG reductions) against the float64 oracle over the first 200 steps
(4 ms, while the activation front crosses the cap): max |dVm| <= 1e-3 * max |Vm|,
AT within one dt, total CG iterations within 2 %."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

STEPS, DT = 200, 0.02


def _mesh():
    from torchcor_b200 import meshgen
    nodes_um, tris = meshgen.icosphere_fast(7, 25.0)
    fib = meshgen.fibres_random_tangent(nodes_um, tris, 7)
    cap = np.nonzero(nodes_um[:, 2] > 24_500.0)[0]
    return nodes_um / 1000.0, tris, np.ones(len(tris), dtype=np.int64), fib, cap


def test_crn_icosphere_level7_float32_vs_float64_oracle(lib, cuda):
    from oracle import port as P
    from torchcor_b200.ionic import CourtemancheRamirezNattel
    from torchcor_b200.simulator import Monodomain
    nodes, tris, reg, fib, cap = _mesh()
    T = STEPS * DT

    ref = P.Monodomain(P.CourtemancheRamirezNattel(DT, dtype=torch.float64), T, DT, dtype=torch.float64)
    ref.load_arrays(nodes, tris, reg, fib)
    ref.add_conductivity([1], il=0.4, it=0.1)
    ref.add_stimulus(torch.from_numpy(cap), 0.0, 2.0, 50, T)
    r = ref.solve(1e-5, 1e-5, 100, snapshot_interval=T / 2)

    sim = Monodomain(CourtemancheRamirezNattel(DT, device=cuda), T=T, dt=DT, device=cuda)
    sim.load_arrays(nodes, tris, reg, fib)
    sim.add_conductivity([1], il=0.4, it=0.1)
    sim.add_stimulus(None, 0.0, 2.0, 50, region=cap)
    sim.solve(1e-5, 1e-5, 100, verbose=False, snapshot_interval=T / 2)

    vm_ref = r.Vm[-1].numpy()
    vm = sim.solutions[-1].cpu().numpy()
    at_ref, at = r.AT.numpy(), sim.activation_time.cpu().numpy()
    assert (at_ref > 0).sum() > 1000                       # the front has moved
    assert np.abs(vm - vm_ref).max() <= 1e-3 * np.abs(vm_ref).max()
    assert np.abs(at - at_ref).max() <= DT * 1.001
    assert abs(sim.n_total_iter - r.n_total_iter) <= max(3, r.n_total_iter // 50)
