"""Generate the golden fixtures of the estimator stage from the reference itself.

Each fixture holds one seeded workload (the arrays of include/upbp_gpu.h, produced by
smallupbp_b200.workload) and the outputs of the reference SmallUPBP estimator code run on it by
the reference harness (oracle/_ref/libupbp_ref.so, built from the reference sources by
oracle/build_ref.py):  per-query PB2D / BB1D (grid and brute force) / PP3D contributions,
per-query candidate counts and hashes, and the splatted image.

The configuration-0 fixture (``config0_cube128``: the 128x128 cube, 16,384 light sub-paths,
r = 0.01, seed 1234) is larger; it stores the reference's outputs and a SHA-256 digest of every
input array instead of the inputs, which the seeded generator recreates (golden_io.load checks the
digests).

Run from the repository root:  python tests/golden/gen_golden.py [fixture names]
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from smallupbp_b200 import workload as W  # noqa: E402
from oracle import ref  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (fixture name, scene config name, overrides)
CASES = [
    ("cube_long_short", "cube32x2048", dict()),
    ("cube_short_long", "cube32x2048", dict(query_beam_type=W.SHORT_BEAM, photon_beam_type=W.LONG_BEAM, seed=77)),
    ("cube_nosine_mindist", "cube24x1536", dict(techniques=W.BPT | W.SURF | W.PP3D | W.PB2D | W.BB1D | W.NO_SINE_IN_WEIGHTS,
                                                min_dist_to_med=0.3, min_path_length=2, max_path_length=5, seed=5)),
    ("cube_previous", "cube24x1536", dict(techniques=W.PP3D | W.PB2D | W.BB1D | W.PREVIOUS | W.BB1D_PREVIOUS, seed=9)),
    ("boxes_all", "boxes", dict()),
    ("cube_wide_radius", "cube24x1536", dict(radius=0.08, seed=21)),
    ("cube_knn_radius", "cube24x1536", dict(radius=0.25, pb2d_knn=8, bb1d_knn=6, seed=31)),
]
# fixtures that keep input digests instead of inputs (regenerated from the config at load time)
DIGEST_CASES = [("config0_cube128", "cube128", dict())]
# the estimators without MIS of VolLightTracer's pure -a pb2d / -a bb1d (W.without_mis: the MIS-only
# inputs are left out, so the C ABI gets NULL for them)
NOMIS_CASES = [
    ("cube_nomis_long", "cube32x2048", dict(radius=0.02, seed=41)),
    ("cube_nomis_short", "cube24x1536", dict(query_beam_type=W.SHORT_BEAM, photon_beam_type=W.SHORT_BEAM,
                                             radius=0.03, seed=43)),
    ("boxes_nomis", "boxes", dict(seed=47)),
]

# the estimator without MIS over the reference's uniform beam grid with the PRESAMPLE beam reduction
# (-gridres, -gridmax, -gridred 0, the evaluator's seed): ref_bb1d and the image follow the grid
GRID_CASES = [
    ("cube_nomis_grid_reduced", "cube32x2048", dict(radius=0.02, seed=41), (32, 2, 0, 1234)),
    ("boxes_nomis_grid_reduced", "boxes", dict(seed=47), (16, 3, 0, 77)),
    ("cube_nomis_grid_short", "cube24x1536", dict(query_beam_type=W.SHORT_BEAM, photon_beam_type=W.SHORT_BEAM,
                                                  radius=0.03, seed=43), (64, 0, 0, 1234)),
    # KNN radii (the reference's kd-tree search): per-beam radii in the rasterisation and the test
    ("cube_nomis_grid_knn", "cube24x1536", dict(radius=0.25, pb2d_knn=8, bb1d_knn=6, seed=53), (24, 3, 0, 99)),
]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()



def scene(name: str, overrides: dict) -> W.SceneConfig:
    if name == "boxes":
        cfg = W.nested_boxes_scene("boxes_small", 24, 24, 2048, 6, 0.02)
    else:
        cfg = W.config(name)
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def main(names=None):
    for fname, cname, over in CASES + DIGEST_CASES + NOMIS_CASES:
        if names and fname not in names:
            continue
        cfg = scene(cname, over)
        w = W.generate(cfg)
        if (fname, cname, over) in NOMIS_CASES:
            w = W.without_mis(w)
        o = ref.run(w, threads=8)
        if (fname, cname, over) in DIGEST_CASES:
            out = {"cfg_name": np.array(cname), "cfg_iteration": np.array(0)}
            out.update({"digest_" + k: np.array(digest(v)) for k, v in w.items()})
        else:
            out = {"in_" + k: v for k, v in w.items()}
        for k in ("pb2d", "bb1d", "bb1d_brute", "pp3d", "count_pb2d", "hash_pb2d", "count_bb1d", "hash_bb1d",
                  "count_pp3d", "hash_pp3d", "image"):
            out["ref_" + k] = o[k]
        if cfg.pb2d_knn > 0 or cfg.bb1d_knn > 0:  # the radii the reference's KNN search produced
            rr = ref.radii(w)
            out["ref_ph_r2"], out["ref_bm_start"], out["ref_bm_end"] = rr["ph_r2"], rr["bm_start"], rr["bm_end"]
        path = os.path.join(HERE, fname + ".npz")
        np.savez_compressed(path, **out)
        print("%-22s lv=%d beams=%d sq=%d pq=%d  cand pb2d=%d bb1d=%d pp3d=%d  %.0f KB" % (
            fname, len(w["lv_path_length"]), len(w["beam_length"]), len(w["sq_path_length"]), len(w["pq_path_length"]),
            o["count_pb2d"].sum(), o["count_bb1d"].sum(), o["count_pp3d"].sum(), os.path.getsize(path) / 1024))

    for fname, cname, over, grid in GRID_CASES:
        if names and fname not in names:
            continue
        cfg = scene(cname, over)
        w = W.without_mis(W.generate(cfg))
        ref.set_grid_options(grid[0], grid[1], grid[2], grid[3])
        try:
            o = ref.run(w, what=ref.PB2D | ref.BB1D_GRID | ref.PP3D, threads=8)
        finally:
            ref.set_grid_options()
        out = {"in_" + k: v for k, v in w.items()}
        out["grid_options"] = np.array(grid, np.int64)
        for k in ("pb2d", "bb1d", "pp3d", "image"):
            out["ref_" + k] = o[k]
        path = os.path.join(HERE, fname + ".npz")
        np.savez_compressed(path, **out)
        print("%-26s grid=%s beams=%d sq=%d  bb1d nonzero=%d  %.0f KB" % (
            fname, grid, len(w["beam_length"]), len(w["sq_path_length"]), int((np.abs(o["bb1d"]).max(1) > 0).sum()),
            os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main(sys.argv[1:] or None)
