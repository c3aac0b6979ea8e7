"""Invariants of the seeded workload generator (the inputs both the oracle and the CUDA path read)."""
import numpy as np
import pytest

from smallupbp_b200 import workload as W


@pytest.fixture(scope="module")
def w():
    return W.generate(W.config("cube24x1536"))


def test_deterministic():
    a = W.generate(W.config("cube16x512"))
    b = W.generate(W.config("cube16x512"))
    assert a.keys() == b.keys()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_light_paths_are_contiguous(w):
    ends = w["lv_path_ends"]
    assert np.all(np.diff(ends) >= 1)  # every path has its light-source vertex
    starts = np.concatenate([[0], ends[:-1]])
    # vertex k of a path has path length k (AccumulateLightPathWeight indexing, PathWeight.hxx:167)
    for p in range(0, len(ends), 97):
        s, e = starts[p], ends[p]
        np.testing.assert_array_equal(w["lv_path_length"][s:e], np.arange(e - s))
        assert np.all(w["lv_path_idx"][s:e] == p)


def test_beams_and_queries_reference_valid_records(w):
    assert np.all(w["beam_light_vertex"] < len(w["lv_path_idx"]))
    assert np.all(w["beam_length"] > 0)
    nseg = len(w["seg_dist_min"])
    assert np.all(w["sq_seg_begin"] + w["sq_seg_count"] <= nseg)
    assert np.all(w["sq_cam_mis_begin"] + w["sq_path_length"] <= len(w["cam_mis"]))
    assert np.all(w["pq_cam_mis_begin"] + w["pq_path_length"] + 1 <= len(w["cam_mis"]))
    assert np.all(w["seg_dist_max"] >= w["seg_dist_min"])
    assert np.all(w["seg_medium"] < len(w["media"]))


def test_iteration_constants_follow_upbp():
    k = W.iteration_constants(W.config("cube128"))
    r, nl = 0.01, 16384
    assert np.isclose(k["eta_pp3d"], 4.0 / 3.0 * np.pi * r ** 3 * nl)
    assert np.isclose(k["eta_pb2d"], np.pi * r * r * nl)
    assert np.isclose(k["eta_bb1d"], 0.5 * r * nl)
