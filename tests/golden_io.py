"""Loading of the golden fixtures (tests/golden/*.npz) and the parity comparison helpers."""
from __future__ import annotations

import glob
import os
from typing import Dict, Tuple

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# fixtures of the reference's uniform beam grid (with its beam reduction): grid_options and the grid's
# outputs only (tests/test_gpu_grid.py); the others hold every estimator's outputs and candidates
GRID_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN_DIR, "*_grid_*.npz")))
FIXTURES = sorted(set(glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))) - set(GRID_FIXTURES))

# Per-query contribution tolerance of the FP32 path against the reference (relative), with an
# absolute floor of ATOL_FRAC times the largest contribution of that estimator in the fixture.
RTOL = 1e-4
ATOL_FRAC = 1e-6


_regenerated: Dict[str, Dict[str, np.ndarray]] = {}


def load(path: str) -> Tuple[Dict[str, np.ndarray], Dict[str, np.ndarray]]:
    """Inputs and reference outputs of a fixture.  A fixture that stores input digests instead of
    inputs (``cfg_name``) is regenerated from its configuration by the seeded generator, and every
    array must match its digest."""
    import hashlib

    from smallupbp_b200.workload import PARAMS_DTYPE

    z = np.load(path)
    if "cfg_name" in z.files:
        if path not in _regenerated:
            from smallupbp_b200 import workload as W

            w = W.generate(W.config(str(z["cfg_name"])), int(z["cfg_iteration"]))
            digests = {k[7:]: str(z[k]) for k in z.files if k.startswith("digest_")}
            assert set(digests) == set(w), "fixture inputs changed: " + str(set(digests) ^ set(w))
            for k, v in w.items():
                got = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
                assert got == digests[k], "the generator no longer reproduces %s of %s" % (k, name(path))
            _regenerated[path] = w
        w = dict(_regenerated[path])
    else:
        w = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    r = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    if w["params"].dtype != PARAMS_DTYPE:  # fixtures written before fields were added: new fields 0
        p = np.zeros(1, PARAMS_DTYPE)
        for f in w["params"].dtype.names:
            p[f] = w["params"][f]
        w["params"] = p
    return w, r


def name(path: str) -> str:
    return os.path.basename(path)[:-4]


def rel_errors(got: np.ndarray, want: np.ndarray) -> np.ndarray:
    """Per-query max-channel relative error with the absolute floor."""
    floor = ATOL_FRAC * max(float(np.abs(want).max()) if want.size else 0.0, 1e-30)
    return (np.abs(got - want) / (np.abs(want) + floor)).max(axis=1)


def assert_close(got: np.ndarray, want: np.ndarray, what: str):
    assert got.shape == want.shape, what
    err = rel_errors(got.astype(np.float64), want.astype(np.float64))
    worst = int(np.argmax(err)) if len(err) else -1
    assert (err <= RTOL).all(), "%s: %d/%d queries above %.0e, worst %.3e at %d (got %s want %s)" % (
        what, int((err > RTOL).sum()), len(err), RTOL, err[worst], worst, got[worst], want[worst])


def image_rel_l2(got: np.ndarray, want: np.ndarray) -> float:
    return float(np.linalg.norm((got - want).ravel()) / max(np.linalg.norm(want.ravel()), 1e-30))


def uses_knn(w: Dict[str, np.ndarray]) -> bool:
    p = w["params"]
    return int(p["pb2d_knn"][0]) > 0 or int(p["bb1d_knn"][0]) > 0


def expected(path: str) -> Tuple[Dict[str, np.ndarray], Dict[str, np.ndarray]]:
    """Workload and the outputs the CUDA path must reproduce: the reference's own (with KNN radii
    too: the default search is the reference's kd-tree search, knn_exact = 0)."""
    return load(path)
