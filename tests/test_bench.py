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
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
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
