"""The bench's reference arm on the CPU: one JSON line with the metric, unit, direction and
workload of the fd3 arm, the CPU baseline it measured and an e2e block with no host-device
traffic (the oracle runs on the host)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("E+F+stress atoms/s")
    assert d["unit"] == "atoms/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    # the arm times a bounded sample of the benchmarked workload and names both
    assert d["config"]["workload"] == "sio2_5184_spme_p5_h1.2_E+F+stress"
    assert d["config"]["sample_of"] == "sio2_139968_spme_p5_h1.2_E+F+stress"
    assert d["config"]["n_atoms"] == 5184
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
