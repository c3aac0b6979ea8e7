"""Autotuner of the estimator stage's launch and structure parameters.

The knobs (``upbp_tuning`` in ``include/upbp_gpu.h``):

* ``bb1d_leaf`` and ``beam_piece_radii`` shape the BB1D beam-piece LBVH: shorter pieces and
  smaller leaves give tighter boxes (fewer tested pieces per query) at the price of more nodes;
* ``bb1d_kernel`` 1 or 2 picks the occupancy the warp-cooperative BB1D gather is compiled for
  (5 or 6 blocks of 4 warps per SM);
* ``pb2d_leaf`` is the photon count per PB2D LBVH leaf;
* ``block_threads`` is the block shape (queries per block) of the thread-per-query PB2D and PP3D
  gathers.

The tuner searches the grids on the caller's own workload, every candidate timed by the
library's per-kernel CUDA events, best of ``repeats``.  The workload stays resident; only the
structures are rebuilt.  Results are plain dicts, so a
caller can store them (``save``/``load``) and skip the search next time for the same workload
signature.
"""
from __future__ import annotations

import itertools
import json
import os
from typing import Dict, Iterable, List, Optional, Tuple


BB1D_SPACE = {"bb1d_leaf": (2, 4, 8), "beam_piece_radii": (2.0, 3.0, 4.0, 6.0), "bb1d_kernel": (1, 2)}
PB2D_SPACE = {"pb2d_leaf": (4, 8, 16), "block_threads": (128, 256)}


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


def autotune(stage, structs, repeats: int = 2, bb1d_space: Optional[Dict] = None,
             pb2d_space: Optional[Dict] = None) -> Tuple[Dict, Dict]:
    """Search the knobs for the workload already loaded into ``stage`` (``EstimatorStage``).

    The BB1D and PB2D knobs are disjoint and each gather's time depends only on its own, so one
    trial times a BB1D candidate and a PB2D candidate together (the shorter list is cycled).
    Each estimator is scored by its gather time; the builds are a few percent of the step.
    Leaves the best tuning set on ``stage`` (built) and returns ``(best, report)``.
    """
    base = stage.get_tuning()
    best = {k: getattr(base, k) for k, _ in base._fields_}
    bb = _grid(bb1d_space or BB1D_SPACE)
    pb = _grid(pb2d_space or PB2D_SPACE)
    trials = []
    score_bb, score_pb = [], []
    for i in range(max(len(bb), len(pb))):
        cand = dict(bb[i % len(bb)], **pb[i % len(pb)])
        stage.set_tuning(**dict(best, **cand))
        t = _time(stage, repeats)
        trials.append(dict(cand, **t))
        if i < len(bb):
            score_bb.append((t["bb1d_ms"], bb[i]))
        if i < len(pb):
            score_pb.append((t["pb2d_ms"], pb[i]))
    best.update(min(score_bb, key=lambda x: x[0])[1])
    best.update(min(score_pb, key=lambda x: x[0])[1])
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
