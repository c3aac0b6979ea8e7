"""Host logic of the multi-GPU path: one process per GPU, two ways to share the work.

**Query shards of one iteration** (``shard_workload``).  The queries of an iteration are
independent once the structures are built, so every rank receives the iteration's whole photon and
beam records, builds the same structures (the builds are deterministic), and evaluates only its
share of the camera queries; one all-reduce (sum) of the framebuffer then gives the iteration's
image.  The shares are 32x32 pixel tiles dealt round-robin with a per-row shift, so every rank
gets tiles all over the image (the cost of a query depends strongly on where its pixel looks).
This makes one iteration faster: strong scaling, with the build repeated on every rank.

**Whole iterations** (``rank_iterations``).  The reference parallelises rendering by iteration
(``SmallUPBP/src/SmallUPBP.cxx:96-131``): every OpenMP thread owns a renderer and runs whole
iterations with its own light pass, acceleration structures and camera pass.  At the end each used
renderer's framebuffer is scaled by 1/its iteration count (``Renderers/Renderer.hxx:55-61``), the
framebuffers are summed and the sum is scaled by 1/(number of renderers used)
(``SmallUPBP.cxx:143-176``).  Here a rank plays the part of a renderer: rank ``r`` of ``W`` runs
iterations ``r, r+W, r+2W, ...`` (each iteration's seed is its index, so the set of iterations does
not depend on ``W``), and the only data-path exchange is the framebuffer combination below: weak
scaling.

Neither mode has anything to exchange inside an iteration, so the framebuffer all-reduce is the
only collective.
"""
from __future__ import annotations

from typing import Dict, List

import numpy as np

SHARD_TILE = 32


def query_shard(pixels: np.ndarray, width: int, rank: int, world: int, tile: int = SHARD_TILE) -> np.ndarray:
    """Indices of the queries that ``rank`` evaluates: the queries whose pixel lies in a tile
    (tile x tile pixels) with (tile row * tiles per row + tile column + tile row) % world == rank.
    Queries without a pixel (pixel < 0) are dealt by their index."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside world size %d" % (rank, world))
    px = np.asarray(pixels, np.int64)
    tiles_x = (width + tile - 1) // tile
    tx, ty = (px % width) // tile, (px // width) // tile
    key = np.where(px >= 0, ty * tiles_x + tx + ty, np.arange(len(px)))
    return np.nonzero(key % world == rank)[0]


def shard_workload(w: Dict[str, np.ndarray], width: int, rank: int, world: int,
                   tile: int = SHARD_TILE) -> Dict[str, np.ndarray]:
    """The workload restricted to ``rank``'s segment and point queries.  Every other array stays
    whole: the photon and beam records (each rank builds the same structures), the volume segments
    and the camera MIS records, which the kept queries index absolutely (``sq_seg_begin``,
    ``*_cam_mis_begin``)."""
    out = dict(w)
    for prefix, key in (("sq_", "sq_pixel"), ("pq_", "pq_pixel")):
        idx = query_shard(w[key], width, rank, world, tile)
        for k, v in w.items():
            if k.startswith(prefix):
                out[k] = np.ascontiguousarray(v[idx])
    return out


def rank_iterations(rank: int, world: int, count: int) -> List[int]:
    """Iteration indices of ``rank``: ``rank + world*j`` for ``j < count``."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside world size %d" % (rank, world))
    return [rank + world * j for j in range(count)]


def split_iterations(total: int, rank: int, world: int) -> List[int]:
    """The rank's share of iterations ``0..total-1`` dealt round-robin (as ``rank_iterations``)."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside world size %d" % (rank, world))
    return list(range(rank, total, world))


def combine_framebuffers(accum, iterations: int, group=None):
    """The reference's final framebuffer from every rank's accumulated one, in place on ``accum``.

    ``accum`` is this rank's sum over its iterations (a torch tensor on the process group's device),
    ``iterations`` how many it ran (0 for a rank that ran none: it does not take part, as an unused
    renderer does not).  Every rank receives the combined framebuffer.
    """
    import torch
    import torch.distributed as dist

    used = 1.0 if iterations > 0 else 0.0
    if iterations > 0:
        accum.mul_(1.0 / iterations)
    else:
        accum.zero_()
    n = torch.tensor([used], dtype=torch.float64, device=accum.device)
    dist.all_reduce(accum, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    n_used = float(n.item())
    if n_used > 0:
        accum.mul_(1.0 / n_used)
    return accum


def max_over_ranks(value: float, device, group=None) -> float:
    """The largest ``value`` of all ranks (the job's time is the slowest rank's)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, device, group=None) -> float:
    """The sum of ``value`` over all ranks (units processed by the whole job)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
