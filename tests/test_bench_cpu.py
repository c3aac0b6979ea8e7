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


def test_reference_arm_reports_samples_not_iterations():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config",
                          "cube16x512", "--steps", "3", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert "samples" in line["steps_are"] and line["ms_per_iteration"] >= line["ms_per_step"]
    assert line["spread"]["min"] <= line["value"] <= line["spread"]["max"]


def test_both_cpu_legs_time_the_same_stratified_sample():
    sys.path.insert(0, ROOT)
    import bench
    from smallupbp_b200 import workload as W

    w = W.make(W.config("cube16x512"))
    a = bench.reference_timing(w, 5, 0, 2)
    b = bench.reference_timing(w, 5, 0, 2)
    assert a["stride"] == b["stride"] >= 1 and a["samples"] == 5
    assert a["sampled_fraction"] == 1.0 / a["stride"]


def test_parity_check_against_the_reference_on_the_oracle():
    """The bench's parity check fed with the C oracle's per-query results (CPU): no mismatches."""
    sys.path.insert(0, ROOT)
    import bench
    from oracle import port
    from smallupbp_b200 import workload as W

    w = W.make(W.config("cube16x512"))
    o = port.run(w)
    res = {"stats": {k: o[k] for k in o if k.startswith(("count_", "hash_"))},
           "pb2d": o["pb2d"], "bb1d": o["bb1d"], "pp3d": o["pp3d"]}
    p = bench.reference_parity(w, {"oracle": res, "absent": None})
    assert p["queries_checked"]["segment"] > 0 and "absent" not in p
    assert p["oracle"]["candidate_mismatches"] == {"pb2d": 0, "bb1d": 0, "pp3d": 0}, p
    for est in ("pb2d", "bb1d", "pp3d"):
        assert p["oracle"]["contributions"][est]["max_rel"] <= 1e-4, p
