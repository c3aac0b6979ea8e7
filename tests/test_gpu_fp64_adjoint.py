"""The FP64 evaluation mode (an FP64 oracle on the GPU) and the adjoint of the estimator sum.

* FP64 mode against the FP64 CPU oracle (oracle/liboracle64.so) on every reference fixture:
  candidate sets bit-exact, per-query contributions equal up to the FP32 rounding of the outputs.
* The adjoint (upbp_adjoint, dual-number kernels) against central finite differences of the FP64
  GPU forward, and against the FP64 reference gradient (central differences of the FP64 CPU
  oracle), within 1e-3 relative.
* The torch.autograd.Function binding (smallupbp_b200.autograd) on an L2 image loss.
"""
import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import engine
from smallupbp_b200 import workload as W

RTOL_GRAD = 1e-3


def _close_per_query(got, want, what, rtol=1e-6):
    g, w = got.astype(np.float64), want.astype(np.float64)
    floor = 1e-6 * max(np.abs(w).max() if w.size else 0.0, 1e-30)
    err = np.abs(g - w) - rtol * np.abs(w)
    assert (err <= floor).all(), "%s: max excess %.3g (floor %.3g)" % (what, err.max() if err.size else 0.0, floor)


@pytest.mark.gpu
@pytest.mark.parametrize("path", G.FIXTURES, ids=G.name)
def test_fp64_mode_matches_fp64_oracle(path):
    from oracle import port

    w, _ = G.load(path)
    o = port.run(w, fp64=True)
    with engine.EstimatorStage(0, engine.MODE_FP64) as st:
        st.run(w)
        pb2d, bb1d = st.segment_results()
        pp3d = st.point_results()
        stats = st.query_stats()
        img = st.image()
    for est in ("pb2d", "bb1d", "pp3d"):
        np.testing.assert_array_equal(stats["count_" + est], o["count_" + est], err_msg=est)
        np.testing.assert_array_equal(stats["hash_" + est], o["hash_" + est], err_msg=est)
    _close_per_query(pb2d, o["pb2d"], "PB2D")
    _close_per_query(bb1d, o["bb1d"], "BB1D")
    _close_per_query(pp3d, o["pp3d"], "PP3D")
    assert G.image_rel_l2(img, o["image"]) <= 1e-6


def _workload():
    return W.generate(W.config("cube32x2048"))


def _loss_weights(n_pix):
    return np.random.default_rng(7).random((n_pix, 3)).astype(np.float32)


def _with_media(media, medium, sa, ss, g):
    m = np.array(media, copy=True)
    m[medium]["absorption"] = sa
    m[medium]["scattering"] = ss
    m[medium]["mean_cosine"] = g
    return m


def _gpu_loss(st, media, wts):
    st.set_media(media)
    st.clear_image()
    st.evaluate()
    return float((st.image().astype(np.float64) * wts).sum())


def _directions(media, medium):
    """(name, function theta -> media) for the grey parameters sigma_a, sigma_s (all channels) and g."""
    m0 = media[medium]
    sa0, ss0, g0 = np.array(m0["absorption"], np.float64), np.array(m0["scattering"], np.float64), float(m0["mean_cosine"])
    return [("sigma_a", sa0[0], lambda t: _with_media(media, medium, sa0 - sa0[0] + t, ss0, g0), slice(0, 3)),
            ("sigma_s", ss0[0], lambda t: _with_media(media, medium, sa0, ss0 - ss0[0] + t, g0), slice(3, 6)),
            ("g", g0, lambda t: _with_media(media, medium, sa0, ss0, t), slice(6, 7))]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [engine.MODE_MIXED, engine.MODE_FP64], ids=["mixed", "fp64"])
def test_adjoint_matches_central_differences_of_fp64_forward(mode):
    import torch

    w = _workload()
    medium = 1
    wts = _loss_weights(w["params"]["image_width"][0] * w["params"]["image_height"][0])
    with engine.EstimatorStage(0, mode) as st:
        st.run(w)
        media = np.array(w["media"], copy=True)
        gi = torch.from_numpy(wts.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)
    with engine.EstimatorStage(0, engine.MODE_FP64) as fd:
        fd.run(w)
        for name, t0, mk, sl in _directions(media, medium):
            h = 1e-3
            d_fd = (_gpu_loss(fd, mk(t0 + h), wts) - _gpu_loss(fd, mk(t0 - h), wts)) / (2 * h)
            d_adj = adj[sl].sum()
            assert abs(d_fd) > 0, name
            assert abs(d_adj - d_fd) <= RTOL_GRAD * abs(d_fd), (name, d_adj, d_fd)


@pytest.mark.gpu
def test_adjoint_per_channel_on_a_non_grey_medium():
    import torch

    w = _workload()
    medium = 1
    w["media"][medium]["absorption"] = (0.05, 0.1, 0.2)   # sigma_t = 0.55, 0.6, 0.7: minimum unambiguous
    wts = _loss_weights(w["params"]["image_width"][0] * w["params"]["image_height"][0])
    media = np.array(w["media"], copy=True)
    with engine.EstimatorStage(0, engine.MODE_FP64) as st:
        st.run(w)
        gi = torch.from_numpy(wts.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)
        sa0, ss0 = np.array(media[medium]["absorption"], np.float64), np.array(media[medium]["scattering"], np.float64)
        g0 = float(media[medium]["mean_cosine"])
        for k in range(7):
            h = 1e-3
            def mk(sign):
                sa, ss, g = sa0.copy(), ss0.copy(), g0
                if k < 3:
                    sa[k] += sign * h
                elif k < 6:
                    ss[k - 3] += sign * h
                else:
                    g += sign * h
                return _with_media(media, medium, sa, ss, g)
            d_fd = (_gpu_loss(st, mk(1), wts) - _gpu_loss(st, mk(-1), wts)) / (2 * h)
            scale = max(abs(d_fd), 1e-3 * np.abs(adj).max())
            assert abs(adj[k] - d_fd) <= 2 * RTOL_GRAD * scale, (k, adj[k], d_fd)


@pytest.mark.gpu
def test_adjoint_matches_fp64_reference_gradient():
    """FP64 reference gradient: central differences of the FP64 CPU oracle."""
    import torch
    from oracle import port

    w = _workload()
    medium = 1
    wts = _loss_weights(w["params"]["image_width"][0] * w["params"]["image_height"][0])
    media = np.array(w["media"], copy=True)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        st.run(w)
        gi = torch.from_numpy(wts.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)

    def cpu_loss(m):
        ww = dict(w)
        ww["media"] = m
        return float((port.run(ww, fp64=True)["image"].astype(np.float64) * wts).sum())

    for name, t0, mk, sl in _directions(media, medium):
        h = 1e-3
        ref = (cpu_loss(mk(t0 + h)) - cpu_loss(mk(t0 - h))) / (2 * h)
        assert abs(adj[sl].sum() - ref) <= RTOL_GRAD * abs(ref), (name, adj[sl].sum(), ref)


@pytest.mark.gpu
def test_autograd_function_l2_loss():
    import torch
    from smallupbp_b200 import autograd

    w = _workload()
    medium = 1
    media = np.array(w["media"], copy=True)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        st.run(w)
        dev = torch.device("cuda")
        tgt = autograd.render(st, media, medium, torch.full((3,), 0.05, dtype=torch.float64, device=dev),
                              torch.full((3,), 0.7, dtype=torch.float64, device=dev),
                              torch.tensor(0.5, dtype=torch.float64, device=dev)).detach().clone()
        sa = torch.full((3,), 0.1, dtype=torch.float64, device=dev, requires_grad=True)
        ss = torch.full((3,), 0.5, dtype=torch.float64, device=dev, requires_grad=True)
        g = torch.tensor(0.3, dtype=torch.float64, device=dev, requires_grad=True)
        img = autograd.render(st, media, medium, sa, ss, g)
        loss = ((img.double() - tgt.double()) ** 2).sum()
        loss.backward()
        grads = (sa.grad.sum().item(), ss.grad.sum().item(), g.grad.item())

        def L(a, s, gg):
            with torch.no_grad():
                im = autograd.render(st, media, medium, torch.full((3,), a, dtype=torch.float64, device=dev),
                                     torch.full((3,), s, dtype=torch.float64, device=dev),
                                     torch.tensor(gg, dtype=torch.float64, device=dev))
                return ((im.double() - tgt.double()) ** 2).sum().item()

        h = 1e-3
        fds = ((L(0.1 + h, 0.5, 0.3) - L(0.1 - h, 0.5, 0.3)) / (2 * h),
               (L(0.1, 0.5 + h, 0.3) - L(0.1, 0.5 - h, 0.3)) / (2 * h),
               (L(0.1, 0.5, 0.3 + h) - L(0.1, 0.5, 0.3 - h)) / (2 * h))
    for a, f in zip(grads, fds):
        assert abs(a - f) <= 5e-3 * abs(f) + 1e-12, (grads, fds)


@pytest.mark.gpu
def test_adjoint_at_config4_size():
    # Configuration 4 at full size: the cube at 512x512 with 262,144 light paths, loss = L2 against
    # the image rendered with sigma_s = 0.7, sigma_a = 0.05, g = 0.5, evaluated at sigma_s = 0.5,
    # sigma_a = 0.1, g = 0.3.  The adjoint (FP32 tangents, FP64 accumulation, mixed-mode structures)
    # against central differences (step 1e-3) of the FP64 GPU forward of the same loss.  (The FP64
    # CPU oracle's gradient is checked at the small size above: its brute-force candidate search
    # over 512^2 queries would take hours.)
    import torch

    w = W.make(W.config("diff512"))
    medium = 1
    media = np.array(w["media"], copy=True)
    tgt_media = _with_media(media, medium, np.full(3, 0.05), np.full(3, 0.7), 0.5)
    with engine.EstimatorStage(0, engine.MODE_FP64) as fd:
        fd.run(w)
        fd.set_media(tgt_media)
        fd.clear_image()
        fd.evaluate()
        target = fd.image().astype(np.float64)
        fd.set_media(media)
        fd.clear_image()
        fd.evaluate()
        img = fd.image().astype(np.float64)
        grad_img = (2.0 * (img - target)).astype(np.float32)

        def loss(m):
            fd.set_media(m)
            fd.clear_image()
            fd.evaluate()
            return float(((fd.image().astype(np.float64) - target) ** 2).sum())

        fds = {}
        for name, t0, mk, sl in _directions(media, medium):
            h = 1e-3
            fds[name] = (loss(mk(t0 + h)) - loss(mk(t0 - h))) / (2 * h)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        st.run(w)
        gi = torch.from_numpy(grad_img.reshape(-1)).cuda()
        torch.cuda.synchronize()
        adj = st.adjoint(gi.data_ptr(), medium)
    for name, t0, mk, sl in _directions(media, medium):
        assert abs(fds[name]) > 0, name
        assert abs(adj[sl].sum() - fds[name]) <= RTOL_GRAD * abs(fds[name]), (name, adj[sl].sum(), fds[name])
