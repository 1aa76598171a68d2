"""bench.py's reference arm on the host cores: one JSON line with the same
metric, unit and workload as the GPU arm, a cpu_baseline record that says
what was timed on how many threads, and an e2e record with no copies."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_contract_line():
    from oracle import refpy
    if not refpy.available():
        pytest.skip("reference oracle not built")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "located pts/s (Newton-resolved, tol 1e-5)"
    assert d["unit"] == "points/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("locate_64: 64^3 hex order 2")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["cores"] >= 1 and cb["threads_used"] == cb["cores"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
