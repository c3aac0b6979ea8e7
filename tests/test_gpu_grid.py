"""BB1D over the reference's uniform beam grid (upbp_set_bb1d_grid) against the reference's own grid
evaluator (Beams/PhGrid.hxx, Beams/Grid.hxx, run by the reference harness): the grid's cells, cell
lists and DDA walk reproduce the reference's, so every query's contribution agrees within 1e-4,
including the pairs that the walk finds in two cells or in none where a closest point falls on a
cell boundary.  With the PRESAMPLE beam reduction (-gridmax, -gridred 0) the same beams are kept
in every over-full cell, which only the reference's own random stream and shuffle give.  The
OFFSET, RESAMPLE_FIXED and SAMPLED reductions draw per query from a stream that does not depend on
the order of evaluation (the reference's depends on it); they are checked for what the reference's
estimators guarantee: averaged over seeds, the estimate of the unreduced grid.
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


def run(stage, w, mode, grid):
    stage.set_mode(mode)
    stage.set_bb1d_grid(*grid)
    try:
        stage.run(w)
        pb2d, bb1d = stage.segment_results()
        return dict(bb1d=bb1d, pb2d=pb2d, image=stage.image(), **stage.query_stats())
    finally:
        stage.set_bb1d_grid(0)


def grid_options(path):
    return tuple(int(x) for x in np.load(path)["grid_options"])


@pytest.mark.gpu
def test_grid_fixtures_present():
    assert len(G.GRID_FIXTURES) >= 3
    assert any(grid_options(p)[1] > 0 for p in G.GRID_FIXTURES)


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.GRID_FIXTURES, ids=G.name)
def test_grid_without_mis_matches_reference(stage, path):
    w, r = G.load(path)
    g = run(stage, w, engine.MODE_PLAIN, grid_options(path))
    G.assert_close(g["bb1d"], r["bb1d"], "BB1D over the reference grid")
    assert G.image_rel_l2(g["image"], r["image"]) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.GRID_FIXTURES, ids=G.name)
def test_grid_mixed_mode_same_candidates(stage, path):
    # mixed mode: the same (cell, beam) pairs as plain FP32; the FP64 closest approach of
    # near-parallel pairs moves only their contributions.  Every query is within 1e-4 of the
    # reference's FP32 grid estimate or, where the grid takes the same pairs as the beam-piece
    # LBVH (same count and hash), of the LBVH's mixed-mode estimate, which the parity tests pin to
    # the FP64 oracle where the reference's FP32 geometry cancels.
    w, r = G.load(path)
    grid = grid_options(path)
    p = run(stage, w, engine.MODE_PLAIN, grid)
    m = run(stage, w, engine.MODE_MIXED, grid)
    lb = run(stage, w, engine.MODE_MIXED, (0, 0, 0, 0))
    np.testing.assert_array_equal(m["count_bb1d"], p["count_bb1d"])
    np.testing.assert_array_equal(m["hash_bb1d"], p["hash_bb1d"])
    got = m["bb1d"].astype(np.float64)
    err = G.rel_errors(got, r["bb1d"].astype(np.float64))
    same = (lb["count_bb1d"] == m["count_bb1d"]) & (lb["hash_bb1d"] == m["hash_bb1d"])
    err = np.where(same, np.minimum(err, G.rel_errors(got, lb["bb1d"].astype(np.float64))), err)
    worst = int(np.argmax(err))
    assert (err <= G.RTOL).all(), (int((err > G.RTOL).sum()), len(err), float(err[worst]), bool(same[worst]))
    assert G.image_rel_l2(m["image"], r["image"]) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_grid_with_mis_matches_reference_grid(stage, path):
    # every fixture holds the reference's grid estimate at its default resolution (-gridres 256) as
    # well as the brute-force one; the two differ where a closest point falls on a cell boundary
    w, r = G.load(path)
    g = run(stage, w, engine.MODE_PLAIN, (256, 0, 0, 1234))
    G.assert_close(g["bb1d"], r["bb1d"], "BB1D over the reference grid (256)")
    G.assert_close(g["pb2d"], r["pb2d"], "PB2D (unchanged by the grid)")


@pytest.mark.gpu
def test_grid_reduction_depends_on_the_seed(stage):
    path = [p for p in G.GRID_FIXTURES if grid_options(p)[1] > 0][0]
    w, r = G.load(path)
    res, mx, red, seed = grid_options(path)
    a = run(stage, w, engine.MODE_PLAIN, (res, mx, red, seed))
    b = run(stage, w, engine.MODE_PLAIN, (res, mx, red, seed + 1))
    full = run(stage, w, engine.MODE_PLAIN, (res, 0, 0, seed))
    G.assert_close(a["bb1d"], r["bb1d"], "reduced, the fixture's seed")
    changed = np.abs(b["bb1d"] - a["bb1d"]).max(1) > 1e-6 * np.abs(a["bb1d"]).max()
    assert changed.mean() > 0.2
    # the reduction tests fewer pairs than the full grid
    assert a["count_bb1d"].sum() < full["count_bb1d"].sum()


@pytest.mark.gpu
def test_grid_options_rejected(stage):
    path = [p for p in G.GRID_FIXTURES if grid_options(p)[1] > 0][0]
    w, _ = G.load(path)
    # reductions beyond SAMPLED, resolutions beyond 1024
    with pytest.raises(engine.UpbpError) as e:
        stage.set_bb1d_grid(32, 2, 4, 1234)
    assert e.value.code == -1
    with pytest.raises(engine.UpbpError):
        stage.set_bb1d_grid(4096)
    # the reduction needs the estimator without MIS
    wm, _ = G.load(G.FIXTURES[0])
    stage.set_mode(engine.MODE_PLAIN)
    stage.set_bb1d_grid(32, 2, 0, 1234)
    try:
        with pytest.raises(engine.UpbpError) as e:
            stage.run(wm)
        assert "without MIS" in str(e.value)
        # the FP64 mode has no grid
        stage.set_mode(engine.MODE_FP64)
        with pytest.raises(engine.UpbpError):
            stage.run(w)
    finally:
        stage.set_bb1d_grid(0)
        stage.set_mode(engine.MODE_PLAIN)
    # and the context still works afterwards
    stage.run(w)


@pytest.mark.gpu
def test_grid_against_the_reference_at_a_larger_size(stage):
    # a 128 x 128 cube iteration without MIS (16,384 light paths), reduced to 4 beams per cell of a
    # 64-cell grid, against the reference harness run here on the same inputs
    from oracle import ref
    from smallupbp_b200 import workload as W

    cfg = W.config("cube128")
    w = W.without_mis(W.generate(cfg, 0))
    grid = (64, 4, 0, 2024)
    ref.set_grid_options(*grid)
    try:
        o = ref.run(w, what=ref.BB1D_GRID, threads=8)
    finally:
        ref.set_grid_options()
    g = run(stage, w, engine.MODE_PLAIN, grid)
    G.assert_close(g["bb1d"], o["bb1d"], "BB1D, reduced grid, cube128")


@pytest.mark.gpu
def test_grid_graph_replay_matches_direct_evaluation():
    # upbp_capture_graph records clear + build + evaluate; the grid build then runs without its host
    # synchronisations, with the sizes of the build before it
    path = [p for p in G.GRID_FIXTURES if grid_options(p)[1] > 0][0]
    w, r = G.load(path)
    s = engine.EstimatorStage(0, engine.MODE_MIXED)
    try:
        s.set_bb1d_grid(*grid_options(path))
        s.run(w)
        _, direct = s.segment_results()
        img = s.image()
        s.capture_graph()
        for _ in range(2):
            s.launch_graph()
            _, replay = s.segment_results()
            np.testing.assert_array_equal(replay, direct)
            assert G.image_rel_l2(s.image(), img) < 1e-6
        G.assert_close(direct, r["bb1d"], "BB1D, reduced grid")
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("reduction", [0, 1, 2, 3], ids=["presample", "offset", "resample_fixed", "sampled"])
def test_grid_reductions_are_unbiased(stage, reduction):
    # every reduction divides a cell's contributions by its selection pdf max_beams / beams, so its
    # mean over seeds is the unreduced grid's estimate; 48 seeds, within 4 standard errors
    path = [p for p in G.GRID_FIXTURES if grid_options(p)[1] > 0][0]
    w, _ = G.load(path)
    res, mx = grid_options(path)[:2]
    f = run(stage, w, engine.MODE_PLAIN, (res, 0, 0, 1))
    full = f["bb1d"].astype(np.float64)
    totals, per_query = [], []
    for seed in range(48):
        g = run(stage, w, engine.MODE_PLAIN, (res, mx, reduction, 1000 + seed))
        assert g["count_bb1d"].sum() < f["count_bb1d"].sum()  # fewer pairs tested and accepted
        per_query.append(g["bb1d"].astype(np.float64))
        totals.append(per_query[-1].sum())
    totals = np.array(totals)
    ref_total = full.sum()
    se = totals.std(ddof=1) / np.sqrt(len(totals))
    assert se > 0, "the seeds changed nothing"
    assert abs(totals.mean() - ref_total) <= 4 * se + 1e-4 * abs(ref_total), (totals.mean(), ref_total, se)
    # and query by query the seed average approaches the unreduced estimate
    mean = np.mean(per_query, axis=0)
    assert G.image_rel_l2(mean, full) < 0.25


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.GRID_FIXTURES, ids=G.name)
def test_grid_structure_bit_exact_with_the_reference(path):
    # the cells' first entries, the beams of every cell in the reference's order (after the build's
    # shuffles) and the selection pdfs, against the reference grid itself (PhGrid.hxx / Grid.hxx)
    from oracle import ref

    w, _ = G.load(path)
    grid = grid_options(path)
    for reduction in ((0, 1) if grid[1] > 0 else (0,)):
        opts = (grid[0], grid[1], reduction, grid[3])
        ref.set_grid_options(*opts)
        try:
            sess = ref.Session(w, what=ref.BB1D_GRID, threads=1)
            want = sess.grid_structure()
            sess.close()
        finally:
            ref.set_grid_options()
        s = engine.EstimatorStage(0, engine.MODE_PLAIN)
        try:
            s.set_bb1d_grid(*opts)
            s.run(w)
            got = s.grid_structure()
        finally:
            s.close()
        np.testing.assert_array_equal(got["cells"], want["cells"])
        np.testing.assert_array_equal(got["beams"], want["beams"])
        if grid[1] > 0:
            np.testing.assert_array_equal(got["pdfs"], want["pdfs"])
        assert want["beams"].size > 0


@pytest.mark.gpu
def test_grid_at_cube512_against_the_reference():
    # configuration-size check: the cube512 iteration (262,144 light paths, 512 x 512, UPBP MIS)
    # over the reference grid at -gridres 64, against the reference harness on the same inputs:
    # the grid structure bit for bit, every query's contribution within 1e-4
    import os
    from oracle import ref
    from smallupbp_b200 import workload as W

    w = W.generate(W.config("cube512"), 0)
    ref.set_grid_options(64, 0, 0, 1234)
    try:
        sess = ref.Session(w, what=ref.BB1D_GRID, threads=os.cpu_count() or 8)
        try:
            want = sess.grid_structure()
            o = sess.eval_outputs(0, 1)
        finally:
            sess.close()
    finally:
        ref.set_grid_options()
    s = engine.EstimatorStage(0, engine.MODE_PLAIN)
    try:
        s.set_bb1d_grid(64)
        s.run(w)
        got = s.grid_structure()
        _, bb1d = s.segment_results()
    finally:
        s.close()
    np.testing.assert_array_equal(got["cells"], want["cells"])
    np.testing.assert_array_equal(got["beams"], want["beams"])
    G.assert_close(bb1d, o["bb1d"], "BB1D over the reference grid, cube512")
