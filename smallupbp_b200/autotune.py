"""Autotuner of the estimator stage's launch and structure parameters.

The knobs (``upbp_tuning`` in ``include/upbp_gpu.h``):

* ``bb1d_leaf`` and ``beam_piece_radii`` shape the BB1D beam-piece LBVH: shorter pieces and
  smaller leaves give tighter boxes (fewer tested pieces per query) at the price of more nodes;
* ``bb1d_kernel`` picks the segment gathers: 1 or 2 the warp-cooperative BB1D kernel compiled for
  6 or 7 blocks of 4 warps per SM (PB2D in its own kernel), 3 or 4 one persistent kernel for all
  camera segments doing PB2D and BB1D per query;
* ``pb2d_kernel`` picks the PB2D gather when it runs on its own: 0 one thread per query, 1 one
  warp per query from a persistent work queue;
* ``pb2d_leaf`` is the photon count per PB2D LBVH leaf;
* ``query_order`` is the order in which the persistent gathers draw the segment queries: 0 along a
  Morton curve of their midpoints, 1 the camera rays by pixel first (neighbouring pixels' rays
  cross nearly the same beam pieces), then the other segments by midpoint;
* ``block_threads`` is the block shape (queries per block) of the thread-per-query PB2D and PP3D
  gathers.

The tuner searches the grids on the caller's own workload, one stage of knobs at a time, every
candidate timed by the library's CUDA events (the whole estimator stage), best of ``repeats``.  The workload stays resident; only the
structures are rebuilt.  Results are plain dicts, so a
caller can store them (``save``/``load``) and skip the search next time for the same workload
signature.
"""
from __future__ import annotations

import itertools
import json
import os
from typing import Dict, Iterable, List, Optional, Tuple


# searched one stage at a time (coordinate descent), each stage a grid over its knobs
STAGES = (
    {"bb1d_kernel": (1, 2, 3, 4)},
    {"bb1d_leaf": (4, 8, 16), "beam_piece_radii": (4.0, 6.0, 8.0), "query_order": (0, 1)},
    {"pb2d_kernel": (0, 1), "pb2d_leaf": (4, 8, 16), "block_threads": (128, 256)},
)


def _grid(space: Dict[str, Iterable]) -> List[Dict]:
    keys = list(space)
    return [dict(zip(keys, vals)) for vals in itertools.product(*(space[k] for k in keys))]


def signature(structs) -> str:
    """Workload signature: sizes and radii that the best parameters depend on."""
    p = structs["params"]
    return "lv%d_b%d_sq%d_pq%d_r%.4g_%.4g_%.4g" % (structs["lv"].n, structs["beams"].n, structs["sq"].n,
                                                  structs["pq"].n, p.radius_pp3d, p.radius_pb2d, p.radius_bb1d)


def _time(stage, repeats: int) -> Dict[str, float]:
    """Per-kernel times (ms) of build + evaluate with the current tuning; best of ``repeats``."""
    stage.build()
    stage.clear_image()
    stage.evaluate()  # warm-up of the freshly built structures
    best: Dict[str, float] = {}
    for _ in range(repeats):
        stage.build()
        stage.clear_image()
        stage.evaluate()
        for k, v in stage.timings().items():
            best[k] = min(best.get(k, float("inf")), v)
    return best


def autotune(stage, structs, repeats: int = 2, stages=STAGES) -> Tuple[Dict, Dict]:
    """Search the knobs for the workload already loaded into ``stage`` (``EstimatorStage``).

    Coordinate descent over ``stages``: each stage times every point of its grid with the best
    values found so far for the other knobs and keeps the fastest.  A candidate's score is the
    whole estimator stage (builds + all gathers) from the library's CUDA events, because the
    fused segment kernel moves PB2D time into the BB1D phase.  Leaves the best tuning set on
    ``stage`` (built) and returns ``(best, report)``.
    """
    base = stage.get_tuning()
    best = {k: getattr(base, k) for k, _ in base._fields_}
    trials = []
    for space in stages:
        scores = []
        for cand in _grid(space):
            stage.set_tuning(**dict(best, **cand))
            t = _time(stage, repeats)
            total = t["build_ms"] + t["pp3d_ms"] + t["pb2d_ms"] + t["bb1d_ms"]
            trials.append(dict(cand, total_ms=total, **t))
            scores.append((total, cand))
        best.update(min(scores, key=lambda x: x[0])[1])
    stage.set_tuning(**best)
    stage.build()
    return best, {"signature": signature(structs), "best": best, "trials": trials}


def save(path: str, report: Dict) -> None:
    data = {}
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[report["signature"]] = report["best"]
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)


def load(path: str, structs) -> Optional[Dict]:
    """The stored best tuning for this workload signature, or None."""
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        return json.load(fh).get(signature(structs))
