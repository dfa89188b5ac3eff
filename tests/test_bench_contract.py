"""The reference arm of bench.py (the oracle timed on the host cores, no GPU
needed) prints one JSON line with the benchmark contract's keys, on the same
metric and workload configuration as the GPU arm."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"],
                       cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    sys.path.insert(0, REPO)
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "cell-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["n_gpus"] == 1 and d["scaling"] == "weak"
    assert abs(d["ms_per_step"] - 1e3 * 128 ** 3 / d["value"]) <= 1e-6 * d["ms_per_step"]
    assert d["config"]["workload"] == "dns128" and d["config"]["grid"] == [128] * 3
    wl = bench.WORKLOADS["dns128"]
    assert d["config"]["nu"] == wl["nu"] and d["config"]["dt"] == wl["dt"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "128^3" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
