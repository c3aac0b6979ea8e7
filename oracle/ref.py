"""Python driver of the reference oracle ``oracle/_ref/libupbp_ref.so`` (test infrastructure only).

The library is the reference SmallUPBP estimator code compiled by ``oracle/build_ref.py``.  Only
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

from smallupbp_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libupbp_ref.so")

PB2D, BB1D_GRID, BB1D_BRUTE, PP3D, CANDIDATES = 1, 2, 4, 8, 16


class RefOutputs(C.Structure):
    _fields_ = [("pb2d_rgb", abi.f32p), ("bb1d_rgb", abi.f32p), ("bb1d_brute_rgb", abi.f32p), ("pp3d_rgb", abi.f32p),
                ("count_pb2d", abi.u32p), ("hash_pb2d", abi.u64p), ("count_bb1d", abi.u32p),
                ("hash_bb1d", abi.u64p), ("count_pp3d", abi.u32p), ("hash_pp3d", abi.u64p), ("image", abi.f32p),
                ("build_ms", C.c_double), ("gather_ms", C.c_double)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(LIB_PATH + " is not built (python oracle/build_ref.py)")
        _lib = C.CDLL(LIB_PATH)
        _lib.ref_run.restype = C.c_int
        _lib.ref_run.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32,
                                 C.POINTER(abi.LightVertices), C.POINTER(abi.Beams), C.POINTER(abi.Mis), C.c_int64,
                                 C.POINTER(abi.SegmentQueries), C.POINTER(abi.PointQueries), C.c_int32, C.c_int64,
                                 C.c_int32, C.POINTER(RefOutputs)]
    return _lib


def run(w: Dict[str, np.ndarray], what: int = PB2D | BB1D_GRID | BB1D_BRUTE | PP3D | CANDIDATES,
        stride: int = 1, threads: int = 0) -> Dict[str, np.ndarray]:
    """Evaluate workload ``w`` with the reference estimator code; returns per-query arrays."""
    s, keep = abi.make_structs(w)
    nq = s["sq"].n
    npq = s["pq"].n
    p = s["params"]
    out: Dict[str, np.ndarray] = {
        "pb2d": np.zeros((nq, 3), np.float32), "bb1d": np.zeros((nq, 3), np.float32),
        "bb1d_brute": np.zeros((nq, 3), np.float32), "pp3d": np.zeros((npq, 3), np.float32),
        "count_pb2d": np.zeros(nq, np.uint32), "hash_pb2d": np.zeros(nq, np.uint64),
        "count_bb1d": np.zeros(nq, np.uint32), "hash_bb1d": np.zeros(nq, np.uint64),
        "count_pp3d": np.zeros(npq, np.uint32), "hash_pp3d": np.zeros(npq, np.uint64),
        "image": np.zeros((p.image_height * p.image_width, 3), np.float32),
    }
    o = RefOutputs(
        pb2d_rgb=abi.ptr(out["pb2d"]), bb1d_rgb=abi.ptr(out["bb1d"]), bb1d_brute_rgb=abi.ptr(out["bb1d_brute"]),
        pp3d_rgb=abi.ptr(out["pp3d"]), count_pb2d=abi.ptr(out["count_pb2d"]), hash_pb2d=abi.ptr(out["hash_pb2d"]),
        count_bb1d=abi.ptr(out["count_bb1d"]), hash_bb1d=abi.ptr(out["hash_bb1d"]),
        count_pp3d=abi.ptr(out["count_pp3d"]), hash_pp3d=abi.ptr(out["hash_pp3d"]), image=abi.ptr(out["image"]))
    rc = lib().ref_run(C.byref(p), s["media"], s["n_media"], C.byref(s["lv"]), C.byref(s["beams"]), s["cam_mis"],
                       s["n_cam_mis"], C.byref(s["sq"]), C.byref(s["pq"]), what, stride, threads, C.byref(o))
    if rc != 0:
        raise RuntimeError("ref_run failed with %d" % rc)
    out["build_ms"] = o.build_ms
    out["gather_ms"] = o.gather_ms
    del keep
    return out
