"""B-P2D (extension): photon beams queried at the camera medium vertices with a 2-D kernel.

The reference has no B-P2D estimator, so the checker is the C restatement's own definition
(oracle/upbp_oracle.c, upbp_oracle_bp2d): parity here is pinned to that definition, not to the
reference.  Candidate sets bit-exact; per-query contributions within the parity tolerance; the
FP64 mode against the FP64 build of the same definition; the adjoint covers B-P2D too.
"""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine
from smallupbp_b200 import workload as W


def _workload(name="cube32x2048", seed_iter=0):
    w = W.generate(W.config(name), iteration=seed_iter)
    w["params"]["techniques"] |= W.BP2D
    return w


def test_oracle_builds_agree_on_candidates():
    from oracle import port

    w = _workload()
    a, b = port.bp2d(w), port.bp2d(w, fp64=True)
    assert a["count_bp2d"].sum() > 100
    np.testing.assert_array_equal(a["count_bp2d"], b["count_bp2d"])
    np.testing.assert_array_equal(a["hash_bp2d"], b["hash_bp2d"])
    # FP32 loses digits where the kernel 1 - d^2/r^2 cancels (points near the kernel edge)
    rel = np.abs(a["bp2d"].astype(np.float64) - b["bp2d"]) / np.maximum(np.abs(b["bp2d"].astype(np.float64)), 1e-30)
    assert np.median(rel[b["bp2d"] != 0]) < 1e-5 and rel.max() < 1e-3
    assert G.image_rel_l2(a["image"], b["image"]) < 1e-4


def test_off_by_default_and_not_a_reference_bit():
    w = W.generate(W.config("cube16x512"))
    assert not (w["params"]["techniques"][0] & W.BP2D)
    assert W.BP2D > 2048  # above every reference flag (SPECULAR_ONLY is 2048)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [engine.MODE_PLAIN, engine.MODE_MIXED], ids=["plain", "mixed"])
@pytest.mark.parametrize("name", ["cube32x2048", "cube64x4096"])
@pytest.mark.parametrize("pb2d_kernel", [0, 1], ids=["thread", "warp"])
def test_gpu_bp2d_matches_oracle(mode, name, pb2d_kernel):
    # pb2d_kernel selects the thread-per-query or the warp-cooperative persistent gather (B-P2D
    # follows the PB2D choice)
    from oracle import port

    w = _workload(name)
    o = port.bp2d(w)
    rest = port.run(w)
    with engine.EstimatorStage(0, mode) as st:
        st.set_tuning(pb2d_kernel=pb2d_kernel)
        st.run(w)
        rgb, cnt, h = st.bp2d_results()
        img = st.image()
    np.testing.assert_array_equal(cnt, o["count_bp2d"])
    np.testing.assert_array_equal(h, o["hash_bp2d"])
    G.assert_close(rgb, o["bp2d"], "B-P2D")
    assert G.image_rel_l2(img, rest["image"] + o["image"]) <= 1e-4


@pytest.mark.gpu
def test_gpu_bp2d_fp64_mode_matches_fp64_oracle():
    from oracle import port

    w = _workload()
    o = port.bp2d(w, fp64=True)
    with engine.EstimatorStage(0, engine.MODE_FP64) as st:
        st.run(w)
        rgb, cnt, h = st.bp2d_results()
    np.testing.assert_array_equal(cnt, o["count_bp2d"])
    g, r = rgb.astype(np.float64), o["bp2d"].astype(np.float64)
    assert (np.abs(g - r) <= 1e-6 * np.abs(r) + 1e-6 * np.abs(r).max()).all()


@pytest.mark.gpu
def test_adjoint_includes_bp2d():
    import torch

    w = _workload()
    medium = 1
    npix = int(w["params"]["image_width"][0] * w["params"]["image_height"][0])
    wts = np.random.default_rng(3).random((npix, 3)).astype(np.float32)
    media = np.array(w["media"], copy=True)
    with engine.EstimatorStage(0, engine.MODE_FP64) as st:
        st.run(w)
        gi = torch.from_numpy(wts.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)

        def loss(g):
            m = np.array(media, copy=True)
            m[medium]["mean_cosine"] = g
            st.set_media(m)
            st.clear_image()
            st.evaluate()
            return float((st.image().astype(np.float64) * wts).sum())

        g0, h = float(media[medium]["mean_cosine"]), 1e-3
        fd = (loss(g0 + h) - loss(g0 - h)) / (2 * h)
    assert abs(adj[6] - fd) <= 1e-3 * abs(fd), (adj[6], fd)
