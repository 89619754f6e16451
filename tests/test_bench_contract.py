"""The reference arm of bench.py (`--impl reference`): the CPU restatement
of the reference path on a bounded sample, printed as one JSON line with the
same metric and workload as the GPU arm and the keys the harness reads.
CPU only: a 4096-row corpus (--rows) keeps it to a few seconds; the default
is the full N = 1,000,000."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_reference_arm():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--rows", "4096"], capture_output=True, text=True, timeout=300, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench

    d = run_reference_arm()
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "queries/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "bn_flat_single_query" and d["config"]["N"] == 4096
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1 and d["vs_baseline"] is None
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "all 4096 rows" in cb["sample"]
    assert cb["value"] == d["value"] > 0
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
