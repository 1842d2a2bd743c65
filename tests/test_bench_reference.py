"""bench.py's reference arm (the CPU oracle on the host cores) keeps the bench line's contract, on CPU and at a
size that finishes in a second: one JSON line with impl, the metric, unit and config of the GPU arm, a
cpu_baseline describing the run, and an e2e with no host-device bytes."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--size", "64", "--steps", "2",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "cell-steps/s"
    assert d["metric"] == "cell-steps/s to 1e-5 rel. residual" and d["higher_is_better"] is True
    assert d["config"] == bench.config_of(64)
    assert d["steps"] == 2 and d["warmup"] == 1 and len(d["pressure_iterations_per_step"]) == 2
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
