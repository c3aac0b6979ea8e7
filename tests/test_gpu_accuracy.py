"""Accuracy at a realistic size: cube512 (512x512 pixels, 262,144 light sub-paths, 217 k segment
and 60 k point queries, 274 M accepted beam pairs).  The plain FP32 and the mixed modes must give
the same candidate sets as the FP64 mode (all three use the reference's FP32 predicates) and an
image within rel-L2 1e-3 of it -- the accuracy bound the throughput is measured at."""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine
from smallupbp_b200 import workload as W

BOUND = 1e-3


@pytest.mark.gpu
def test_full_size_images_within_the_bound_of_fp64():
    w = W.generate(W.config("cube512"), 0)
    imgs, stats = {}, {}
    for m in (engine.MODE_PLAIN, engine.MODE_MIXED, engine.MODE_FP64):
        with engine.EstimatorStage(0, m) as st:
            st.run(w)
            imgs[m], stats[m] = st.image(), st.query_stats()
    ref = imgs[engine.MODE_FP64]
    assert np.abs(ref).sum() > 0
    for m in (engine.MODE_PLAIN, engine.MODE_MIXED):
        for k in stats[m]:
            np.testing.assert_array_equal(stats[m][k], stats[engine.MODE_FP64][k], err_msg=k)
        l2 = G.image_rel_l2(imgs[m], ref)
        assert l2 <= BOUND, (m, l2)
