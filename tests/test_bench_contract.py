"""bench.py's reference arm on a tiny workload (CPU only): it prints one JSON
line with the keys the benchmark contract asks for."""
from __future__ import annotations

import json
import os
import subprocess
import sys
import time

from conftest import ROOT


def test_reference_arm_json_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--points", "3000",
           "--views", "2", "--res", "64x64", "--steps", "2", "--warmup", "3"]
    t0 = time.perf_counter()
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    wall = time.perf_counter() - t0
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 3
    assert d["unit"] == "train-steps/s" and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
    # the line states the work it timed: its sampled steps fit in the run's wall time
    assert d["steps"] * d["ms_per_step"] / 1e3 <= wall
    assert d["full_step_ms_estimate"] > 0
