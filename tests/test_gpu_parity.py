"""Parity of the CUDA estimator stage with the reference SmallUPBP estimator code.

The fixtures hold seeded workloads and the outputs of the reference's own EmbreeBre::evalBre,
PhotonBeamsEvaluator::evalBeamBeamEstimate (USE_BRUTE and USE_GRID) and HashGrid::Process with
UPBP::RangeQuery (tests/golden/gen_golden.py).  Candidate sets must match bit-exactly (count and
order-independent hash per query); per-query contributions within 1e-4 relative.
"""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine


@pytest.fixture(scope="module")
def stage():
    s = engine.EstimatorStage(0, engine.MODE_PLAIN)
    yield s
    s.close()


def run(stage, w, mode=engine.MODE_PLAIN):
    stage.set_mode(mode)
    stage.run(w)
    pb2d, bb1d = stage.segment_results()
    return dict(pb2d=pb2d, bb1d=bb1d, pp3d=stage.point_results(), image=stage.image(), **stage.query_stats())


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_candidate_sets_bit_exact(stage, path):
    w, r = G.expected(path)
    g = run(stage, w)
    for est in ("pb2d", "bb1d", "pp3d"):
        np.testing.assert_array_equal(g["count_" + est], r["count_" + est], err_msg=est + " candidate counts")
        np.testing.assert_array_equal(g["hash_" + est], r["hash_" + est], err_msg=est + " candidate hashes")


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_contributions_plain_fp32(stage, path):
    w, r = G.expected(path)
    g = run(stage, w)
    G.assert_close(g["pb2d"], r["pb2d"], "PB2D")
    G.assert_close(g["bb1d"], r["bb1d_brute"], "BB1D vs brute-force reference")
    G.assert_close(g["pp3d"], r["pp3d"], "PP3D")
    assert G.image_rel_l2(g["image"], r["image"]) <= 1e-4


@pytest.mark.gpu
def test_deterministic_candidates_and_stable_image(stage):
    w, _ = G.load(G.FIXTURES[0])
    a = run(stage, w)
    b = run(stage, w)
    for k in ("count_pb2d", "hash_pb2d", "count_bb1d", "hash_bb1d", "count_pp3d", "hash_pp3d", "pp3d"):
        np.testing.assert_array_equal(a[k], b[k])
    assert G.image_rel_l2(a["image"], b["image"]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_mixed_mode_candidates_and_contributions(stage, path):
    # Mixed mode: same FP32 candidate predicates (bit-exact sets), FP64 MIS partial sums and an FP64
    # closest-approach solve for near-parallel beam pairs.  Every query's contribution is within
    # 1e-4 of the FP32 reference or, where the reference's own FP32 geometry cancels, of the FP64
    # oracle (the same candidates, FP64 arithmetic); the image agrees within 1e-4 rel L2.
    from oracle import port

    w, r = G.expected(path)
    g = run(stage, w, engine.MODE_MIXED)
    for est in ("pb2d", "bb1d", "pp3d"):
        np.testing.assert_array_equal(g["hash_" + est], r["hash_" + est], err_msg=est)
    o64 = port.run(w, fp64=True)
    for est, rk in (("pb2d", "pb2d"), ("bb1d", "bb1d_brute"), ("pp3d", "pp3d")):
        got = g[est].astype(np.float64)
        err = np.minimum(G.rel_errors(got, r[rk].astype(np.float64)), G.rel_errors(got, o64[est].astype(np.float64)))
        worst = int(np.argmax(err)) if len(err) else -1
        assert (err <= G.RTOL).all(), (est, int((err > G.RTOL).sum()), float(err[worst]) if worst >= 0 else None)
    assert G.image_rel_l2(g["image"], r["image"]) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_image_error_against_fp64_oracle(stage, path):
    # Both modes within 1e-3 image rel L2 of the FP64 oracle (same candidates, FP64 arithmetic).
    from oracle import port
    w, _ = G.load(path)
    o64 = port.run(w, fp64=True)
    for mode in (engine.MODE_PLAIN, engine.MODE_MIXED):
        g = run(stage, w, mode)
        assert G.image_rel_l2(g["image"], o64["image"]) <= 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4],
                         ids=["thread_per_query", "warp5", "warp6", "segments5", "segments6"])
@pytest.mark.parametrize("leaf", [1, 4, 16])
def test_bb1d_kernel_variants_same_candidates(stage, kernel, leaf):
    # Every BB1D gather variant and every leaf size / piece length finds the reference's
    # candidate set (and the fused segment kernel the PB2D one as well).
    w, r = G.load(G.FIXTURES[-1])
    stage.set_tuning(bb1d_kernel=kernel, bb1d_leaf=leaf, beam_piece_radii=4.0 if leaf == 16 else 8.0)
    try:
        g = run(stage, w)
        np.testing.assert_array_equal(g["count_bb1d"], r["count_bb1d"])
        np.testing.assert_array_equal(g["hash_bb1d"], r["hash_bb1d"])
        np.testing.assert_array_equal(g["count_pb2d"], r["count_pb2d"])
        np.testing.assert_array_equal(g["hash_pb2d"], r["hash_pb2d"])
        G.assert_close(g["bb1d"], r["bb1d_brute"], "BB1D")
        G.assert_close(g["pb2d"], r["pb2d"], "PB2D")
    finally:
        stage.set_tuning(bb1d_kernel=2, bb1d_leaf=8, beam_piece_radii=6.0)


@pytest.mark.gpu
@pytest.mark.parametrize("pb2d_kernel", [0, 1], ids=["thread", "warp"])
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_pb2d_kernel_variants_same_candidates(stage, pb2d_kernel, path):
    # the thread-per-query and the warp-cooperative persistent PB2D gathers find the reference's
    # candidate set (the oracle's for KNN radii), in plain FP32 with the reference's contributions
    w, r = G.expected(path)
    stage.set_tuning(pb2d_kernel=pb2d_kernel, bb1d_kernel=2)
    try:
        g = run(stage, w)
        np.testing.assert_array_equal(g["count_pb2d"], r["count_pb2d"])
        np.testing.assert_array_equal(g["hash_pb2d"], r["hash_pb2d"])
        G.assert_close(g["pb2d"], r["pb2d"], "PB2D")
    finally:
        stage.set_tuning(pb2d_kernel=1)


@pytest.mark.gpu
@pytest.mark.parametrize("knn_exact", [0, 1], ids=["reference_search", "exact"])
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED], ids=["plain", "mixed"])
def test_knn_radii_bit_exact_with_the_oracle(stage, mode, knn_exact):
    # KNN radii at a size where photons and beam origins span many tree levels: with knn_exact = 0
    # the CUDA kd-tree search must return what the reference's search returns (the oracle's
    # restatement of it is pinned to the reference's own radii), with knn_exact = 1 the exact k-th
    # nearest distance; either way the candidate sets match the oracle's bit for bit (PB2D, BB1D and
    # B-P2D).
    from oracle import port
    from smallupbp_b200 import workload as W

    cfg = W.config("cube64x4096")
    cfg.radius, cfg.pb2d_knn, cfg.bb1d_knn = 0.3, 10, 7
    w = W.generate(cfg)
    w["params"]["techniques"] |= W.BP2D
    w["params"]["knn_exact"] = knn_exact
    o = port.run(w)
    ob = port.bp2d(w)
    g = run(stage, w, mode)
    for est in ("pb2d", "bb1d", "pp3d"):
        np.testing.assert_array_equal(g["count_" + est], o["count_" + est], err_msg=est)
        np.testing.assert_array_equal(g["hash_" + est], o["hash_" + est], err_msg=est)
    if mode == engine.MODE_PLAIN:
        G.assert_close(g["pb2d"], o["pb2d"], "PB2D (KNN)")
        G.assert_close(g["bb1d"], o["bb1d"], "BB1D (KNN)")
    rgb, cnt, h = stage.bp2d_results()
    np.testing.assert_array_equal(cnt, ob["count_bp2d"])
    np.testing.assert_array_equal(h, ob["hash_bp2d"])
    assert G.image_rel_l2(g["image"], o["image"] + ob["image"]) <= 1e-4


@pytest.mark.gpu
def test_knn_reference_search_at_cube512(stage):
    # The reference's KNN search on 10^5-point sets: the top levels of the kd-tree are partitioned
    # block-parallel (segments of more than 4096 points), then one warp per segment, the smallest
    # one thread per segment.  A sample of the queries (every 97th) must see the oracle's candidate
    # sets, which follow the reference's radii.
    from oracle import port
    from smallupbp_b200 import workload as W

    cfg = W.config("cube512")
    cfg.pb2d_knn, cfg.bb1d_knn = 12, 8
    w = W.generate(cfg)
    assert int((w["lv_flags"] & 1).sum()) > 50_000 and len(w["beam_length"]) > 50_000
    o = port.run(w, stride=97)
    g = run(stage, w, engine.MODE_MIXED)
    q = np.arange(0, len(g["count_bb1d"]), 97)
    for est in ("pb2d", "bb1d"):
        np.testing.assert_array_equal(g["count_" + est][q], o["count_" + est][q], err_msg=est)
        np.testing.assert_array_equal(g["hash_" + est][q], o["hash_" + est][q], err_msg=est)
    qp = np.arange(0, len(g["count_pp3d"]), 97)
    np.testing.assert_array_equal(g["hash_pp3d"][qp], o["hash_pp3d"][qp])
