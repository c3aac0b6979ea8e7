"""bench.py's CPU legs: the reference arm's JSON line and the CPU baseline (all cores and one core),
on a small workload.  They run the reference's estimator code built into oracle/_ref, so they skip
where that library was not built."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_available():
    sys.path.insert(0, ROOT)
    from oracle import ref
    return ref.available()


pytestmark = pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built")


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config",
                          "cube16x512", "--steps", "2", "--warmup", "1", "--cpu-seconds", "0.5"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "queries/s"
    assert line["steps"] == 2 and line["warmup"] == 1 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["cores"] >= 1 and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_cpu_baseline_reports_all_cores_and_one_core():
    sys.path.insert(0, ROOT)
    import bench
    from smallupbp_b200 import workload as W

    base = bench.cpu_baseline(W.make(W.config("cube16x512")), 0.5)
    assert base["kind"] == "reference" and base["cores"] >= 1 and base["value"] > 0
    assert base["one_core"]["value"] > 0 and base["one_core"]["ms_per_iteration"] > 0
