"""bench.py's reference arm runs on the host cores (no GPU): one JSON line
with the GPU arm's metric, unit and direction, "impl": "reference", a
cpu_baseline describing the run (kind, cores, sample; value = the line's),
and an e2e block with the line's value and no host<->device bytes. Run on
the ams40 workload (a 40^3 PCG solve of the restatement takes about a second
here; the default eddy64 workload's full 64^3 COCR solve takes minutes)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "ams40",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is False and line["n_gpus"] == 1 and line["steps"] == 1
    assert line["value"] > 0 and line["config"]["workload"].startswith("ams40")
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"]
    e = line["e2e"]
    assert e["value"] == line["value"] and e["unit"] == line["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
