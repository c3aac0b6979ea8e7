"""The estimator stage as a differentiable function of one medium's parameters.

``EstimatorImage.apply(sigma_a, sigma_s, g, stage, media, medium)`` returns the framebuffer that
``upbp_evaluate`` accumulates (``[H*W][3]`` float32 on the current CUDA device) for the workload
already loaded, built and queried on ``stage`` (an ``engine.EstimatorStage`` in mixed or FP64
mode), with ``media[medium]`` replaced by the given ``sigma_a`` (3), ``sigma_s`` (3) and ``g``.
The backward pass calls ``upbp_adjoint``: the hand-written adjoint kernels recompute every
candidate's contribution with forward-mode tangents (transmittance is recomputed, not stored)
and contract them with the incoming framebuffer gradient.

What is differentiated: everything the estimators compute from the media table -- transmittance
along the query and the beam, the ray-sampling pdfs, sigma_s, the Henyey-Greenstein phase
function and the MIS weights' medium-dependent terms -- with every other input (paths, photons,
beams, camera records, candidate sets) held fixed.  The index of the smallest sigma_t component
is a discrete choice and is held at its value; for a grey medium (equal sigma_t in all channels)
move the channels together (scalar sigma_s and sigma_a broadcast to rgb) so that it does not
switch.
"""
from __future__ import annotations

import numpy as np
import torch


class EstimatorImage(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma_a, sigma_s, g, stage, media, medium):
        m = np.array(media, copy=True)
        m[medium]["absorption"] = sigma_a.detach().double().cpu().numpy()
        m[medium]["scattering"] = sigma_s.detach().double().cpu().numpy()
        m[medium]["mean_cosine"] = float(g.detach().cpu())
        stage.set_media(m)
        stage.clear_image()
        stage.evaluate()
        dev = sigma_a.device if sigma_a.is_cuda else torch.device("cuda")
        img = torch.empty(stage.pixels() * 3, dtype=torch.float32, device=dev)
        torch.cuda.synchronize(dev)
        stage.read_image_into(img.data_ptr())
        ctx.stage, ctx.media, ctx.medium = stage, m, medium
        ctx.devices = (sigma_a.device, sigma_s.device, g.device)
        return img.view(-1, 3)

    @staticmethod
    def backward(ctx, grad_img):
        stage = ctx.stage
        stage.set_media(ctx.media)  # the parameters of this forward pass
        gi = grad_img.detach().to(torch.float32).contiguous()
        if not gi.is_cuda:
            gi = gi.cuda()
        torch.cuda.synchronize(gi.device)
        d = stage.adjoint(gi.data_ptr(), ctx.medium)
        da, ds, dg = ctx.devices
        return (torch.tensor(d[0:3], dtype=torch.float64, device=da), torch.tensor(d[3:6], dtype=torch.float64, device=ds),
                torch.tensor(d[6], dtype=torch.float64, device=dg), None, None, None)


def render(stage, media, medium, sigma_a, sigma_s, g):
    """Differentiable framebuffer ([H*W][3]) for one medium's parameters."""
    return EstimatorImage.apply(sigma_a, sigma_s, g, stage, media, medium)
