"""The estimators without MIS: VolLightTracer's pure PB2D and BB1D (`-a pb2d`, `-a bb1d`).

VolLightTracer builds EmbreeBre over VltLightVertex records, so its photons take the callback
breIntersectFuncHomogeneous (Bre/Bre.cxx:239-291), and calls evalBeamBeamEstimate without
AdditionalRayDataForMis, which takes PhotonBeam::accumulate (Beams/PhotonBeam.hxx:315-367)
(Renderers/VolLightTracer.hxx:296-412).  The fixtures cube_nomis_long, cube_nomis_short and
boxes_nomis hold the reference harness's outputs for those calls; their workloads leave every
MIS-only input out, so the C ABI receives NULL for them.  Candidate sets must match bit for bit and
per-query contributions within 1e-4 relative, for every gather variant and mode.
"""
import ctypes as C

import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import abi, engine
from smallupbp_b200 import workload as W

NOMIS = [p for p in G.FIXTURES if "nomis" in G.name(p)]


@pytest.fixture(scope="module")
def stage():
    s = engine.EstimatorStage(0, engine.MODE_PLAIN)
    yield s
    s.close()


def run(stage, w, mode):
    stage.set_mode(mode)
    stage.run(w)
    pb2d, bb1d = stage.segment_results()
    return dict(pb2d=pb2d, bb1d=bb1d, image=stage.image(), **stage.query_stats())


def test_fixtures_present():
    assert len(NOMIS) == 3
    for p in NOMIS:
        w, _ = G.load(p)
        assert int(w["params"]["techniques"][0]) & W.NO_MIS
        assert not set(W.MIS_ONLY_INPUTS) & set(w)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4],
                         ids=["thread_per_query", "warp6", "warp7", "segments5", "segments6"])
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED, engine.MODE_FP64],
                         ids=["plain", "mixed", "fp64"])
@pytest.mark.parametrize("path", NOMIS, ids=G.name)
def test_nomis_matches_reference(stage, path, mode, kernel):
    # Plain FP32: every query within 1e-4 of the reference.  Mixed mode solves near-parallel beam
    # pairs in FP64 and the FP64 mode everything: every query within 1e-4 of the FP32 reference or,
    # where the reference's FP32 geometry cancels, of the FP64 oracle.
    from oracle import port

    w, r = G.load(path)
    stage.set_tuning(bb1d_kernel=kernel, pb2d_kernel=0 if kernel == 0 else 1)
    try:
        g = run(stage, w, mode)
    finally:
        stage.set_tuning(bb1d_kernel=2, pb2d_kernel=1)
    for est in ("pb2d", "bb1d"):
        np.testing.assert_array_equal(g["count_" + est], r["count_" + est], err_msg=est + " candidate counts")
        np.testing.assert_array_equal(g["hash_" + est], r["hash_" + est], err_msg=est + " candidate hashes")
    assert r["count_pb2d"].sum() > 100 and r["count_bb1d"].sum() > 1000
    if mode == engine.MODE_PLAIN:
        G.assert_close(g["pb2d"], r["pb2d"], "PB2D without MIS")
        G.assert_close(g["bb1d"], r["bb1d_brute"], "BB1D without MIS")
    else:
        o64 = port.run(w, fp64=True)
        for est, rk in (("pb2d", "pb2d"), ("bb1d", "bb1d_brute")):
            got = g[est].astype(np.float64)
            err = np.minimum(G.rel_errors(got, r[rk].astype(np.float64)),
                             G.rel_errors(got, o64[est].astype(np.float64)))
            assert (err <= G.RTOL).all(), (est, float(err.max()))
    assert G.image_rel_l2(g["image"], r["image"]) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("path", NOMIS, ids=G.name)
def test_nomis_fp64_mode_matches_fp64_oracle(stage, path):
    from oracle import port

    w, _ = G.load(path)
    o64 = port.run(w, fp64=True)
    g = run(stage, w, engine.MODE_FP64)
    for est in ("pb2d", "bb1d"):
        err = G.rel_errors(g[est].astype(np.float64), o64[est].astype(np.float64))
        assert err.max() <= G.RTOL, (est, float(err.max()))
    assert G.image_rel_l2(g["image"], o64["image"]) <= 1e-6


@pytest.mark.gpu
def test_nomis_contributions_differ_from_mis_and_skip_rejects(stage):
    # The same workload with MIS: the weights change the contributions, and without MIS the
    # path-length rejects of accumulate2 / breIntersectFuncHomogeneous2 do not apply.
    path = next(p for p in G.FIXTURES if G.name(p) == "cube_long_short")
    w, r = G.load(path)
    wn = W.without_mis(w)
    g = run(stage, wn, engine.MODE_PLAIN)
    np.testing.assert_array_equal(g["hash_bb1d"], r["hash_bb1d"])
    np.testing.assert_array_equal(g["hash_pb2d"], r["hash_pb2d"])
    assert np.abs(g["bb1d"]).sum() > np.abs(r["bb1d_brute"]).sum()
    assert np.abs(g["pb2d"]).sum() > np.abs(r["pb2d"]).sum()


@pytest.mark.gpu
def test_mis_inputs_required_with_mis(stage):
    # Only UPBP_NO_MIS may leave the MIS inputs out: with MIS the build and evaluate fail loudly.
    path = next(p for p in G.FIXTURES if G.name(p) == "cube_long_short")
    w, _ = G.load(path)
    for drop in ("lv_mis", "beam_light_vertex"):
        w2 = dict(w)
        del w2[drop]
        stage.load(w2)
        with pytest.raises(engine.UpbpError) as e:
            stage.build()
        assert e.value.code == -1
    w2 = dict(w)
    del w2["sq_cam_mis_begin"]
    stage.load(w2)
    stage.build()
    stage.set_queries(w2)
    with pytest.raises(engine.UpbpError) as e:
        stage.evaluate()
    assert e.value.code == -1


@pytest.mark.gpu
def test_nomis_with_pp3d_is_rejected(stage):
    w, _ = G.load(NOMIS[0])
    s, keep = abi.make_structs(w)
    p = s["params"]
    p.techniques |= W.PP3D
    rc = stage._l.upbp_set_params(stage._ctx, C.byref(p))
    assert rc == -1
    del keep


@pytest.mark.gpu
def test_nomis_adjoint_matches_central_differences():
    # The adjoint of the estimator sum without MIS (the same Dual-number gathers) against central
    # differences of the FP64 forward, grey sigma_a, sigma_s and g of the scattering medium.
    import torch
    from test_gpu_fp64_adjoint import RTOL_GRAD, _directions, _gpu_loss, _loss_weights

    w = W.without_mis(W.generate(W.config("cube32x2048")))
    medium = 1
    wts = _loss_weights(w["params"]["image_width"][0] * w["params"]["image_height"][0])
    media = np.array(w["media"], copy=True)
    with engine.EstimatorStage(0, engine.MODE_FP64) as st:
        st.run(w)
        gi = torch.from_numpy(wts.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)
        for name, t0, mk, sl in _directions(media, medium):
            h = 1e-3
            d_fd = (_gpu_loss(st, mk(t0 + h), wts) - _gpu_loss(st, mk(t0 - h), wts)) / (2 * h)
            assert abs(d_fd) > 0, name
            assert abs(adj[sl].sum() - d_fd) <= RTOL_GRAD * abs(d_fd), (name, adj[sl].sum(), d_fd)
