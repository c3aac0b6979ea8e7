"""Python driver of the oracle's C restatement ``oracle/liboracle.so`` (test infrastructure only).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict

import numpy as np

from smallupbp_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")      # FP32 restatement
LIB64_PATH = os.path.join(HERE, "liboracle64.so")  # FP64 oracle
_libs = {}


def lib(fp64: bool = False):
    path = LIB64_PATH if fp64 else LIB_PATH
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(path + " is not built (python oracle/build_oracle.py)")
        l = C.CDLL(path)
        l.upbp_oracle_run.restype = C.c_int
        l.upbp_oracle_run.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32,
                                         C.POINTER(abi.LightVertices), C.POINTER(abi.Beams), C.POINTER(abi.Mis),
                                         C.POINTER(abi.SegmentQueries), C.POINTER(abi.PointQueries), C.c_int64,
                                         abi.f32p, abi.f32p, abi.f32p, abi.u32p, abi.u64p, abi.u32p, abi.u64p,
                                         abi.u32p, abi.u64p, abi.f32p]
        _libs[path] = l
    return _libs[path]


def run(w: Dict[str, np.ndarray], stride: int = 1, fp64: bool = False, radii=None,
        reach: bool = True) -> Dict[str, np.ndarray]:
    """Evaluate workload ``w`` with the C restatement (``fp64``: the FP64 oracle build).

    ``radii`` = (photon radius^2 per light vertex, beam start radius, beam end radius) replaces the
    KNN search (used to inject the radii the reference's own builds produced).  ``reach``: apply the
    BB1D reach rule that defines the CUDA path's candidate set (off: the reference's brute-force
    candidate set, which also holds pairs the FP32 predicate accepts only through rounding)."""
    s, keep = abi.make_structs(w)
    l = lib(fp64)
    l.upbp_oracle_set_reach.restype = None
    l.upbp_oracle_set_reach.argtypes = [C.c_int]
    l.upbp_oracle_set_reach(1 if reach else 0)
    l.upbp_oracle_set_radii.restype = None
    l.upbp_oracle_set_radii.argtypes = [abi.f32p] * 3
    if radii is not None:
        radii = [np.ascontiguousarray(a, np.float32) for a in radii]
        l.upbp_oracle_set_radii(*[abi.ptr(a) for a in radii])
    else:
        l.upbp_oracle_set_radii(None, None, None)
    nq, npq = s["sq"].n, s["pq"].n
    p = s["params"]
    out = {"pb2d": np.zeros((nq, 3), np.float32), "bb1d": np.zeros((nq, 3), np.float32),
           "pp3d": np.zeros((npq, 3), np.float32), "count_pb2d": np.zeros(nq, np.uint32),
           "hash_pb2d": np.zeros(nq, np.uint64), "count_bb1d": np.zeros(nq, np.uint32),
           "hash_bb1d": np.zeros(nq, np.uint64), "count_pp3d": np.zeros(npq, np.uint32),
           "hash_pp3d": np.zeros(npq, np.uint64),
           "image": np.zeros((p.image_width * p.image_height, 3), np.float32)}
    P = abi.ptr
    rc = lib(fp64).upbp_oracle_run(C.byref(p), s["media"], s["n_media"], C.byref(s["lv"]), C.byref(s["beams"]),
                               s["cam_mis"], C.byref(s["sq"]), C.byref(s["pq"]), stride, P(out["pb2d"]),
                               P(out["bb1d"]), P(out["pp3d"]), P(out["count_pb2d"]), P(out["hash_pb2d"]),
                               P(out["count_bb1d"]), P(out["hash_bb1d"]), P(out["count_pp3d"]), P(out["hash_pp3d"]),
                               P(out["image"]))
    l.upbp_oracle_set_radii(None, None, None)
    l.upbp_oracle_set_reach(1)
    if rc != 0:
        raise RuntimeError("upbp_oracle_run failed (%d)" % rc)
    del keep, radii
    return out


def bp2d(w: Dict[str, np.ndarray], stride: int = 1, fp64: bool = False) -> Dict[str, np.ndarray]:
    """B-P2D (extension) of workload ``w`` with the C restatement: per point query rgb, count, hash,
    and the framebuffer of the B-P2D contributions alone."""
    s, keep = abi.make_structs(w)
    l = lib(fp64)
    f = l.upbp_oracle_bp2d
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32, C.POINTER(abi.Beams),
                  C.POINTER(abi.PointQueries), C.c_int64, abi.f32p, abi.u32p, abi.u64p, abi.f32p]
    npq = s["pq"].n
    p = s["params"]
    out = {"bp2d": np.zeros((npq, 3), np.float32), "count_bp2d": np.zeros(npq, np.uint32),
           "hash_bp2d": np.zeros(npq, np.uint64), "image": np.zeros((p.image_width * p.image_height, 3), np.float32)}
    P = abi.ptr
    rc = f(C.byref(p), s["media"], s["n_media"], C.byref(s["beams"]), C.byref(s["pq"]), stride, P(out["bp2d"]),
           P(out["count_bp2d"]), P(out["hash_bp2d"]), P(out["image"]))
    if rc != 0:
        raise RuntimeError("upbp_oracle_bp2d failed (%d)" % rc)
    del keep
    return out


def knn_radii(w: Dict[str, np.ndarray], fp64: bool = False) -> Dict[str, np.ndarray]:
    """The KNN radii of the oracle's builds for workload ``w`` (``params.knn_exact`` picks the
    reference's kd-tree search or the exact k-th nearest distance): photon radius^2 per light
    vertex, beam start and end radius."""
    s, keep = abi.make_structs(w)
    l = lib(fp64)
    l.upbp_oracle_knn_radii.restype = C.c_int
    l.upbp_oracle_knn_radii.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.LightVertices), C.POINTER(abi.Beams),
                                        abi.f32p, abi.f32p, abi.f32p]
    out = {"ph_r2": np.zeros(s["lv"].n, np.float32), "bm_start": np.zeros(s["beams"].n, np.float32),
           "bm_end": np.zeros(s["beams"].n, np.float32)}
    rc = l.upbp_oracle_knn_radii(C.byref(s["params"]), C.byref(s["lv"]), C.byref(s["beams"]), abi.ptr(out["ph_r2"]),
                                 abi.ptr(out["bm_start"]), abi.ptr(out["bm_end"]))
    if rc != 0:
        raise RuntimeError("upbp_oracle_knn_radii failed (%d)" % rc)
    del keep
    return out
