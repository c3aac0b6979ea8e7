"""The autotuner: search-space bookkeeping on CPU; on the GPU, a search on a reference fixture whose
chosen tuning must keep the candidate sets bit-exact and the contributions within tolerance."""
import json

import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import abi, autotune, engine


def test_grid_enumerates_the_product():
    g = autotune._grid({"a": (1, 2), "b": (3.0, 4.0, 5.0)})
    assert len(g) == 6
    assert {"a": 2, "b": 4.0} in g


def test_save_and_load_by_signature(tmp_path):
    w, _ = G.load(G.FIXTURES[0])
    s, keep = abi.make_structs(w)
    path = str(tmp_path / "tuning.json")
    assert autotune.load(path, s) is None
    best = {"pb2d_leaf": 8, "bb1d_leaf": 2, "block_threads": 128, "beam_piece_radii": 4.0, "bb1d_kernel": 1}
    autotune.save(path, {"signature": autotune.signature(s), "best": best, "trials": []})
    assert autotune.load(path, s) == best
    with open(path) as fh:
        assert list(json.load(fh)) == [autotune.signature(s)]
    del keep


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED], ids=["plain", "mixed"])
def test_autotuned_stage_keeps_parity(mode):
    w, r = G.load(G.FIXTURES[0])
    with engine.EstimatorStage(0, mode) as st:
        s = st.load(w)
        st.set_queries(w)
        best, rep = autotune.autotune(st, s, repeats=1,
                                      stages=({"bb1d_kernel": (0, 1, 3)},
                                              {"bb1d_leaf": (1, 8), "beam_piece_radii": (4.0, 16.0)},
                                              {"pb2d_leaf": (4, 16), "block_threads": (64,)}))
        assert len(rep["trials"]) == 3 + 4 + 2
        assert best["bb1d_leaf"] in (1, 8) and best["pb2d_leaf"] in (4, 16)
        t = st.get_tuning()
        assert (t.bb1d_leaf, t.pb2d_leaf, t.block_threads) == (best["bb1d_leaf"], best["pb2d_leaf"], 64)
        st.clear_image()
        st.evaluate()
        pb2d, bb1d = st.segment_results()
        stats = st.query_stats()
    for est in ("pb2d", "bb1d"):
        np.testing.assert_array_equal(stats["count_" + est], r["count_" + est])
        np.testing.assert_array_equal(stats["hash_" + est], r["hash_" + est])
    if mode == engine.MODE_PLAIN:
        G.assert_close(pb2d, r["pb2d"], "PB2D after autotuning")
        G.assert_close(bb1d, r["bb1d_brute"], "BB1D after autotuning")
