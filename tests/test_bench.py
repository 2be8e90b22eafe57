"""bench.py on the CPU: the reference arm's JSON line (the oracle timed on the host
cores) on the small Mitchell-Schaeffer cube, warm-up steps run untimed."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_time_oracle_runs_warmup_untimed():
    sys.path.insert(0, str(ROOT))
    import bench
    from torchcor_b200.workloads import ms_cube
    r = bench.time_oracle(ms_cube(), budget_s=0.0, min_steps=2, max_steps=2, warmup=3)
    assert r["steps"] == 2 and r["warmup"] == 3
    assert r["value"] > 0 and r["seconds"] > 0


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "ms_cube", "--steps", "2",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "node-steps/s" and line["higher_is_better"]
    assert line["steps"] == 2 and line["warmup"] == 3 and line["value"] > 0
    # the reference itself where it is installed under baseline/_ref, else the oracle
    kind = "reference" if (ROOT / "baseline" / "_ref" / "torchcor").is_dir() else "port"
    assert line["cpu_baseline"]["kind"] == kind and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "node-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] and line["config"]["nodes"] == 9261


def test_clock_sampler_counts_marked_segments_only():
    sys.path.insert(0, str(ROOT))
    import bench
    c = bench.ClockSampler(0)
    c.proc = False                                   # no nvidia-smi here: feed samples by hand
    line = "0, {}, 1965, 500, 0x0, Not Active, Not Active, Not Active, {}"
    c.segments = [["headline", 1.0, 2.0], ["e2e", 3.0, 4.0]]
    c.samples = [(0.5, line.format(300, "Not Active")), (1.5, line.format(1965, "Not Active")),
                 (2.5, line.format(300, "Not Active")), (3.5, line.format(1900, "Active"))]
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == (1965 + 1900) / 2 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"] and set(s["segments"]) == {"headline", "e2e"}


def test_reference_harness_matches_oracle_steps():
    """The bench's reference harness (the reference's own Monodomain.step with the
    oracle's matrices) takes the same steps as the oracle, bit for bit."""
    import pytest
    import torch
    sys.path.insert(0, str(ROOT))
    import bench
    from torchcor_b200.workloads import ms_cube
    if bench.import_reference() is None:
        pytest.skip("reference not installed under baseline/_ref")
    wl = ms_cube()
    ref = bench.ReferenceRun(wl)
    sim, u = ref.build("cpu")
    osim = bench.oracle_sim(wl)
    osim.assemble()
    v = osim.ionic.initialize(osim.n_nodes)
    osim.cg.initialize(v, linear_guess=True)
    t = 0.0
    for _ in range(40):
        t += wl.dt
        u, it, _, _ = sim.step(u, t, 1e-5, 1e-5, 100)
        v, it2 = osim.step(v, t, 1e-5, 1e-5, 100)
        assert it == it2
    assert torch.equal(u, v)
