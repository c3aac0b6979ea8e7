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
        _lib.ref_set_grid_options.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        _lib.ref_set_grid_options.restype = None
        _lib.ref_set_grid_seed.argtypes = [C.c_int32]
        _lib.ref_set_grid_seed.restype = None
    return _lib


def set_grid_options(grid_size: int = 256, max_beams_in_cell: int = 0, reduction_type: int = 0,
                     seed: int = 1234) -> None:
    """The reference's -gridres / -gridmax / -gridred options (defaults 256, 0, 0) and the grid
    evaluator's reduction seed (PhotonBeamsEvaluator::mSeed, default 1234)."""
    lib().ref_set_grid_options(grid_size, max_beams_in_cell, reduction_type)
    lib().ref_set_grid_seed(seed)


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


class Session:
    """Reference structures built once (one world per thread, as the reference keeps one renderer
    per OpenMP thread); ``eval(offset, stride)`` runs the reference estimators on a query subset."""

    def __init__(self, w: Dict[str, np.ndarray], what: int = PB2D | BB1D_GRID | PP3D, threads: int = 0):
        l = lib()
        l.ref_prepare.restype = C.c_void_p
        l.ref_prepare.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32,
                                  C.POINTER(abi.LightVertices), C.POINTER(abi.Beams), C.POINTER(abi.Mis),
                                  C.POINTER(abi.SegmentQueries), C.POINTER(abi.PointQueries), C.c_int32, C.c_int32]
        l.ref_eval.restype = C.c_int
        l.ref_eval.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(RefOutputs)]
        l.ref_release.argtypes = [C.c_void_p]
        self._l = l
        self._s, self._keep = abi.make_structs(w)
        s = self._s
        self.n_segment = s["sq"].n
        self.n_point = s["pq"].n
        self._h = l.ref_prepare(C.byref(s["params"]), s["media"], s["n_media"], C.byref(s["lv"]),
                                C.byref(s["beams"]), s["cam_mis"], C.byref(s["sq"]), C.byref(s["pq"]), what, threads)
        if not self._h:
            raise RuntimeError("ref_prepare failed")
        o = RefOutputs()
        self._l.ref_eval(self._h, max(self.n_segment, self.n_point), 1, C.byref(o))  # no queries: reads the build time
        self.build_ms = o.build_ms

    def grid_structure(self) -> Dict[str, np.ndarray]:
        """The reference grid's cell lists (a session prepared with BB1D_GRID): ``cells`` (mCells),
        ``beams`` (mPointers as beam indices) and ``pdfs`` (mPdfs)."""
        l = self._l
        l.ref_grid_structure.restype = C.c_int
        l.ref_grid_structure.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        nc, ne = C.c_int64(), C.c_int64()
        if l.ref_grid_structure(self._h, None, None, None, C.byref(nc), C.byref(ne)) != 0:
            raise RuntimeError("ref_grid_structure failed")
        cells = np.zeros(nc.value, np.uint32)
        beams = np.zeros(ne.value, np.int32)
        pdfs = np.zeros(max(nc.value - 1, 0), np.float32)
        l.ref_grid_structure(self._h, cells.ctypes.data, beams.ctypes.data, pdfs.ctypes.data, C.byref(nc), C.byref(ne))
        return {"cells": cells, "beams": beams, "pdfs": pdfs}

    def eval(self, offset: int, stride: int) -> float:
        """Evaluate queries offset, offset+stride, ...; returns the wall time in ms."""
        o = RefOutputs()
        rc = self._l.ref_eval(self._h, offset, stride, C.byref(o))
        if rc != 0:
            raise RuntimeError("ref_eval failed")
        return o.gather_ms

    def eval_outputs(self, offset: int, stride: int) -> Dict[str, np.ndarray]:
        """Evaluate queries offset, offset+stride, ... and return their per-query outputs (rows of
        the other queries stay zero) and ``gather_ms``.  Candidate counts and hashes are filled when
        the session was prepared with CANDIDATES."""
        nq, npq = self.n_segment, self.n_point
        out = {"pb2d": np.zeros((nq, 3), np.float32), "bb1d": np.zeros((nq, 3), np.float32),
               "bb1d_brute": np.zeros((nq, 3), np.float32), "pp3d": np.zeros((npq, 3), np.float32),
               "count_pb2d": np.zeros(nq, np.uint32), "hash_pb2d": np.zeros(nq, np.uint64),
               "count_bb1d": np.zeros(nq, np.uint32), "hash_bb1d": np.zeros(nq, np.uint64),
               "count_pp3d": np.zeros(npq, np.uint32), "hash_pp3d": np.zeros(npq, np.uint64)}
        o = RefOutputs(
            pb2d_rgb=abi.ptr(out["pb2d"]), bb1d_rgb=abi.ptr(out["bb1d"]), bb1d_brute_rgb=abi.ptr(out["bb1d_brute"]),
            pp3d_rgb=abi.ptr(out["pp3d"]), count_pb2d=abi.ptr(out["count_pb2d"]), hash_pb2d=abi.ptr(out["hash_pb2d"]),
            count_bb1d=abi.ptr(out["count_bb1d"]), hash_bb1d=abi.ptr(out["hash_bb1d"]),
            count_pp3d=abi.ptr(out["count_pp3d"]), hash_pp3d=abi.ptr(out["hash_pp3d"]))
        rc = self._l.ref_eval(self._h, offset, stride, C.byref(o))
        if rc != 0:
            raise RuntimeError("ref_eval failed")
        out["gather_ms"] = o.gather_ms
        return out

    def close(self):
        if self._h:
            self._l.ref_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radii(w: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """The photon and beam radii the reference's own builds assign to workload ``w`` (KNN or
    constant): per light vertex the photon radius^2 (0 for non-photons), per beam the start and end
    radius and the max radius^2."""
    s, keep = abi.make_structs(w)
    l = lib()
    l.ref_prepare.restype = C.c_void_p
    l.ref_prepare.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32, C.POINTER(abi.LightVertices),
                              C.POINTER(abi.Beams), C.POINTER(abi.Mis), C.POINTER(abi.SegmentQueries),
                              C.POINTER(abi.PointQueries), C.c_int32, C.c_int32]
    l.ref_radii.restype = C.c_int
    l.ref_radii.argtypes = [C.c_void_p] + [abi.f32p] * 4
    l.ref_release.argtypes = [C.c_void_p]
    h = l.ref_prepare(C.byref(s["params"]), s["media"], s["n_media"], C.byref(s["lv"]), C.byref(s["beams"]),
                      s["cam_mis"], C.byref(s["sq"]), C.byref(s["pq"]), PB2D | BB1D_BRUTE, 1)
    if not h:
        raise RuntimeError("ref_prepare failed")
    nlv, nb = s["lv"].n, s["beams"].n
    out = {"ph_r2": np.zeros(nlv, np.float32), "bm_start": np.zeros(nb, np.float32),
           "bm_end": np.zeros(nb, np.float32), "bm_r2": np.zeros(nb, np.float32)}
    rc = l.ref_radii(h, *[abi.ptr(out[k]) for k in ("ph_r2", "bm_start", "bm_end", "bm_r2")])
    l.ref_release(h)
    del keep
    if rc != 0:
        raise RuntimeError("ref_radii failed")
    return out
