"""bench.py's reference arm, run on the host cores (no GPU): one JSON line with the metric, its unit and
direction, the workload, a CPU baseline describing the run, and an end-to-end figure with no host-device copies."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_line():
    lib = os.path.join(ROOT, "oracle", "_ref", "libqed_ref.so")
    if not os.path.exists(lib):
        pytest.fail("the reference engine library is not built (oracle/Makefile, run by __graft_entry__.build())")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "H.v/s" and d["unit"] == "H.v/s"
    assert d["higher_is_better"] is True and d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3
    assert d["config"]["workload"] and d["config"]["dim"] == 252091362
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
