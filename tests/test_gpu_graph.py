"""CUDA graph of the estimator stage (upbp_capture_graph / upbp_launch_graph): a replay of
clear + build + evaluate gives the per-query results of the direct calls bit for bit (one warp or
thread per query, fixed traversal order) and the same framebuffer up to the order of the splat
atomics; every upload discards the graph."""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine


def _results(st):
    pb2d, bb1d = st.segment_results()
    return pb2d, bb1d, st.point_results(), st.query_stats(), st.image()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED, engine.MODE_FP64], ids=["plain", "mixed", "fp64"])
def test_graph_replay_matches_direct_calls(mode):
    import torch

    w, r = G.load(G.FIXTURES[0])
    stream = torch.cuda.Stream()
    with engine.EstimatorStage(0, mode) as st:
        st.set_stream(stream.cuda_stream)
        st.run(w)
        want = _results(st)
        st.capture_graph()
        for _ in range(2):  # replays are repeatable
            st.clear_image()  # zeroes the framebuffer and every per-query result
            assert not _results(st)[1].any()
            st.launch_graph()
            got = _results(st)
            for a, b in zip(got[:3], want[:3]):
                np.testing.assert_array_equal(a, b)
            for k in got[3]:
                np.testing.assert_array_equal(got[3][k], want[3][k])
            assert G.image_rel_l2(got[4], want[4]) < 1e-6
    for est in ("pb2d", "bb1d", "pp3d"):
        np.testing.assert_array_equal(want[3]["count_" + est], r["count_" + est])


@pytest.mark.gpu
def test_upload_discards_the_graph():
    import torch

    w, _ = G.load(G.FIXTURES[0])
    stream = torch.cuda.Stream()
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        st.set_stream(stream.cuda_stream)
        with pytest.raises(engine.UpbpError):
            st.capture_graph()  # nothing built yet
        st.run(w)
        st.capture_graph()
        st.launch_graph()
        st.set_media(w["media"])
        with pytest.raises(engine.UpbpError) as e:
            st.launch_graph()
        assert e.value.code == -4
        st.build()
        st.clear_image()
        st.evaluate()
        st.capture_graph()
        st.launch_graph()
        st.set_tuning(bb1d_leaf=2)
        with pytest.raises(engine.UpbpError):
            st.launch_graph()
