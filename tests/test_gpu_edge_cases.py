"""Edge cases of the C-ABI path on small and empty inputs: no beams, one beam, a sparse subset of
beams, no segment queries, no point queries.  The candidates the change leaves alone stay the full
workload's; the results follow the oracle (the C restatement, under the same reach rule and the
reference's MIS rules) and, over the reference grid, the reference's own grid."""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine


@pytest.fixture(scope="module")
def stage():
    s = engine.EstimatorStage(0, engine.MODE_PLAIN)
    yield s
    s.close()


def run(stage, w, mode=engine.MODE_PLAIN, grid=None):
    stage.set_mode(mode)
    if grid:
        stage.set_bb1d_grid(*grid)
    try:
        stage.run(w)
        pb2d, bb1d = stage.segment_results()
        return dict(pb2d=pb2d, bb1d=bb1d, pp3d=stage.point_results(), image=stage.image(), **stage.query_stats())
    finally:
        if grid:
            stage.set_bb1d_grid(0)


def with_beams(w, idx):
    out = dict(w)
    for k, v in w.items():
        if k.startswith("beam_"):
            out[k] = np.ascontiguousarray(v[idx])
    return out


def without(w, prefixes):
    out = dict(w)
    for k, v in w.items():
        if any(k.startswith(p) for p in prefixes):
            out[k] = np.ascontiguousarray(v[:0])
    return out


def workload():
    # the first MIS fixture (a 32x32 cube iteration, 2,048 light paths), without KNN radii
    path = [p for p in G.FIXTURES if not G.uses_knn(G.load(p)[0])][0]
    return G.load(path)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED], ids=["plain", "mixed"])
def test_no_beams(stage, mode):
    # the PB2D and PP3D candidates stay; their MIS weights change, because without beams the
    # renderer passes no beam evaluator (UPBP.hxx:780, :885 pass NULL for an empty beam array) and
    # the BB1D selection pdf of the candidates is 0 (Bre.cxx:407): the oracle follows the same rule
    from oracle import port

    w = workload()
    full = run(stage, w, mode)
    wn = with_beams(w, np.zeros(0, np.int64))
    o = port.run(wn)
    for grid in (None, (64, 0, 0, 1234)):
        e = run(stage, wn, mode, grid)
        assert not e["bb1d"].any() and int(e["count_bb1d"].sum()) == 0
        for est in ("pb2d", "pp3d"):
            np.testing.assert_array_equal(e["hash_" + est], full["hash_" + est])
            np.testing.assert_array_equal(e["hash_" + est], o["hash_" + est])
            G.assert_close(e[est], o[est], est + " without beams")


def with_knn(w):
    # KNN radii from the reference's kd-tree search (8 photons, 6 beam origins)
    out = dict(w)
    p = np.array(w["params"], copy=True)
    p["pb2d_knn"], p["bb1d_knn"], p["knn_exact"] = 8, 6, 0
    out["params"] = p
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("knn", [False, True], ids=["constant_radius", "knn_radii"])
@pytest.mark.parametrize("subset", ["one", "two", "sparse"])
def test_few_beams_match_the_oracle(stage, subset, knn):
    # with KNN radii this covers the kd-tree over one and two beam origins and a small tree
    from oracle import port

    w = with_knn(workload()) if knn else workload()
    nb = len(w["beam_length"])
    if subset in ("one", "two"):
        # the beam with the most accepted pairs in the full workload (by the oracle), and its successor
        counts = [int(port.run(with_beams(w, np.array([k])))["count_bb1d"].sum()) for k in range(0, nb, max(1, nb // 64))]
        idx = np.array([int(np.argmax(counts)) * max(1, nb // 64)])
        if subset == "two":
            idx = np.array([idx[0], (idx[0] + 1) % nb])
    else:
        idx = np.arange(0, nb, 97)
    ws = with_beams(w, idx)
    o = port.run(ws)
    g = run(stage, ws)
    assert int(o["count_bb1d"].sum()) > 0
    np.testing.assert_array_equal(g["count_bb1d"], o["count_bb1d"])
    np.testing.assert_array_equal(g["hash_bb1d"], o["hash_bb1d"])
    G.assert_close(g["bb1d"], o["bb1d"], "BB1D with %d beams" % len(idx))


@pytest.mark.gpu
def test_sparse_beams_over_the_reference_grid(stage):
    from oracle import ref

    w = workload()
    ws = with_beams(w, np.arange(0, len(w["beam_length"]), 97))
    ref.set_grid_options(16, 0, 0, 1234)
    try:
        o = ref.run(ws, what=ref.BB1D_GRID, threads=4)
    finally:
        ref.set_grid_options()
    g = run(stage, ws, grid=(16, 0, 0, 1234))
    assert np.abs(o["bb1d"]).max() > 0
    G.assert_close(g["bb1d"], o["bb1d"], "BB1D over the reference grid, sparse beams")


@pytest.mark.gpu
def test_no_segment_queries_and_no_point_queries(stage):
    w = workload()
    full = run(stage, w)
    e = run(stage, without(w, ("sq_", "seg_")))
    assert e["bb1d"].shape[0] == 0 and e["pb2d"].shape[0] == 0
    np.testing.assert_array_equal(e["hash_pp3d"], full["hash_pp3d"])
    np.testing.assert_array_equal(e["pp3d"], full["pp3d"])
    e = run(stage, without(w, ("pq_",)))
    assert e["pp3d"].shape[0] == 0
    for est in ("pb2d", "bb1d"):
        np.testing.assert_array_equal(e["hash_" + est], full["hash_" + est])
        np.testing.assert_array_equal(e[est], full[est])
    # neither kind: the image stays black
    e = run(stage, without(w, ("sq_", "seg_", "pq_")))
    assert not e["image"].any()
