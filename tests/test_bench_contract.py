"""The reference arm of bench.py (`--impl reference`): the CPU restatement
of the reference path on a bounded sample, printed as one JSON line with the
same metric and workload as the GPU arm and the keys the harness reads.
CPU only (a 512-row sample keeps it well under a second)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_reference_arm():
    env = dict(os.environ, BN_CPU_SAMPLE_ROWS="512")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench

    d = run_reference_arm()
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "queries/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "bn_flat_single_query" and d["config"]["N"] == 1_000_000
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1 and d["vs_baseline"] is None
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "512 rows" in cb["sample"]
    assert cb["value"] == d["value"] > 0
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
