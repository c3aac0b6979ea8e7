"""The BB1D candidate set does not depend on the acceleration structure.

The beam-piece LBVH changes with the leaf size, the piece length and the gather kernel the
autotuner picks, and every BB1D kernel applies the same reach rule (a pair the reference's FP32
predicate accepts is kept when the FP64 distance of the segments is within the radius at their
closest point plus 2e-5 + 1e-3 r).  So every tuning must give the same per-query candidate counts and
order-independent hashes: on configuration 0 (128x128 cube, 16,384 light sub-paths, r = 0.01)
equal to the reference's own estimators, and on cube512 (217 k segment queries, 274 M accepted
pairs) equal across tunings and modes."""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine
from smallupbp_b200 import workload as W

TUNINGS = [
    dict(bb1d_kernel=2, bb1d_leaf=8, beam_piece_radii=6.0),
    dict(bb1d_kernel=1, bb1d_leaf=4, beam_piece_radii=4.0),
    dict(bb1d_kernel=3, bb1d_leaf=16, beam_piece_radii=8.0),
    dict(bb1d_kernel=4, bb1d_leaf=2, beam_piece_radii=3.0),
    dict(bb1d_kernel=0, bb1d_leaf=8, beam_piece_radii=12.0),
]


def _stats(w, mode, tuning):
    with engine.EstimatorStage(0, mode) as st:
        st.set_tuning(**tuning)
        st.run(w)
        return st.query_stats()


@pytest.mark.gpu
def test_config0_candidates_equal_reference_for_every_tuning():
    path = next(p for p in G.FIXTURES if G.name(p) == "config0_cube128")
    w, r = G.load(path)
    for tun in TUNINGS:
        s = _stats(w, engine.MODE_MIXED, tun)
        for est in ("pb2d", "bb1d", "pp3d"):
            np.testing.assert_array_equal(s["count_" + est], r["count_" + est], err_msg="%s %s" % (est, tun))
            np.testing.assert_array_equal(s["hash_" + est], r["hash_" + est], err_msg="%s %s" % (est, tun))


@pytest.mark.gpu
def test_cube512_candidates_identical_across_tunings_and_modes():
    w = W.generate(W.config("cube512"), 0)
    base = _stats(w, engine.MODE_MIXED, TUNINGS[0])
    assert base["count_bb1d"].astype(np.int64).sum() > 100_000_000
    for mode, tun in [(engine.MODE_MIXED, t) for t in TUNINGS[1:]] + [(engine.MODE_PLAIN, TUNINGS[1]),
                                                                      (engine.MODE_FP64, TUNINGS[0])]:
        s = _stats(w, mode, tun)
        for k in ("count_bb1d", "hash_bb1d"):
            diff = int((s[k] != base[k]).sum())
            assert diff == 0, (k, mode, tun, diff)
