"""bench.py's command line: the options that select other measurements than the default line."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _parse(argv):
    old = sys.argv
    sys.argv = ["bench.py"] + argv
    try:
        return bench.parse()
    finally:
        sys.argv = old


def test_defaults_measure_everything_on_one_gpu():
    a = _parse([])
    assert a.gpus == 1 and a.impl == "b200" and a.config == "cube1024" and a.mode == "mixed"
    assert a.warmup >= 3 and a.bb1d_grid == 0
    assert not (a.no_e2e or a.no_arms or a.no_parity or a.no_secondary or a.no_accuracy)


def test_grid_option_keeps_only_the_measurements_defined_for_it():
    # BB1D over the reference grid: the e2e, accuracy, device-pass, arm, parity and secondary
    # measurements are defined for the LBVH path and are skipped; the tuning is the library's
    a = _parse(["--bb1d-grid", "64"])
    assert a.bb1d_grid == 64 and a.no_autotune
    assert a.no_e2e and a.no_accuracy and a.no_device_passes and a.no_arms and a.no_parity and a.no_secondary


def test_dropin_is_the_plain_thread_per_query_gather():
    import json
    a = _parse(["--dropin"])
    assert a.mode == "plain" and a.no_autotune
    t = json.loads(a.tuning)
    assert t["bb1d_kernel"] == 0 and t["pb2d_kernel"] == 0


def test_knn_option_names_the_two_neighbour_counts():
    a = _parse(["--knn", "8,6"])
    assert a.knn == "8,6"
    assert tuple(int(x) for x in a.knn.split(",")) == (8, 6)
