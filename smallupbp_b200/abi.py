"""ctypes mirror of ``include/upbp_gpu.h`` and helpers that point its structs at numpy arrays.

A workload is a dict of numpy arrays (see :mod:`smallupbp_b200.workload`).  :func:`make_structs`
returns the C structs for it together with the list of arrays they reference (keep it alive while
the structs are in use).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Tuple

import numpy as np

from .workload import MEDIUM_DTYPE, MIS_DTYPE, PARAMS_DTYPE

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
i64p = C.POINTER(C.c_int64)
u64p = C.POINTER(C.c_uint64)


class Medium(C.Structure):
    _fields_ = [("absorption", C.c_float * 3), ("scattering", C.c_float * 3), ("mean_cosine", C.c_float),
                ("continuation_prob", C.c_float)]


class Mis(C.Structure):
    _fields_ = [(n, C.c_float) for n in MIS_DTYPE.names[:-1]] + [("flags", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [(n, C.c_uint32 if PARAMS_DTYPE[n].kind == "u" else (C.c_int32 if PARAMS_DTYPE[n].kind == "i" else C.c_float))
                for n in PARAMS_DTYPE.names]


class LightVertices(C.Structure):
    _fields_ = [("n", C.c_int64), ("position", f32p), ("throughput", f32p), ("dir_fix", f32p), ("cont_prob", f32p),
                ("path_idx", i32p), ("path_length", i32p), ("medium_id", i32p), ("flags", u32p),
                ("mis", C.POINTER(Mis)), ("n_paths", C.c_int32), ("path_ends", i32p)]


class Beams(C.Structure):
    _fields_ = [("n", C.c_int64), ("origin", f32p), ("direction", f32p), ("length", f32p), ("throughput", f32p),
                ("flags", u32p), ("ray_sample_pdf", f32p), ("ray_sample_rev_pdf", f32p),
                ("ray_sampling_flags", u32p), ("last_pdf_w_inv", f32p), ("medium_id", i32p), ("light_vertex", i32p)]


class SegmentQueries(C.Structure):
    _fields_ = [("n", C.c_int64), ("origin", f32p), ("direction", f32p), ("seg_begin", i32p), ("seg_count", i32p),
                ("flags", u32p), ("path_length", i32p), ("last_pdf_w_inv", f32p), ("throughput", f32p),
                ("pixel", i32p), ("cam_mis_begin", i64p), ("n_segments", C.c_int64), ("seg_dist_min", f32p),
                ("seg_dist_max", f32p), ("seg_pdf", f32p), ("seg_rev_pdf", f32p), ("seg_attenuation", f32p),
                ("seg_medium", i32p)]


class PointQueries(C.Structure):
    _fields_ = [("n", C.c_int64), ("position", f32p), ("dir_fix", f32p), ("medium_id", i32p),
                ("path_length", i32p), ("throughput", f32p), ("pixel", i32p), ("cam_mis_begin", i64p)]


class Tuning(C.Structure):
    _fields_ = [("pb2d_leaf", C.c_int32), ("bb1d_leaf", C.c_int32), ("block_threads", C.c_int32),
                ("beam_piece_radii", C.c_float), ("bb1d_kernel", C.c_int32), ("pb2d_kernel", C.c_int32),
                ("query_order", C.c_int32)]


class Bb1dGrid(C.Structure):
    """upbp_bb1d_grid: the reference's uniform beam grid (-gridres, -gridmax, -gridred, mSeed)."""
    _fields_ = [("grid_res", C.c_uint32), ("max_beams_in_cell", C.c_uint32), ("reduction", C.c_uint32),
                ("seed", C.c_int32)]


class QueryStats(C.Structure):
    _fields_ = [("count_pb2d", u32p), ("hash_pb2d", u64p), ("count_bb1d", u32p), ("hash_bb1d", u64p),
                ("count_pp3d", u32p), ("hash_pp3d", u64p)]


MAX_BOXES, SCENE_MAX_MEDIA = 8, 16


class SceneMedium(C.Structure):
    _fields_ = [("absorption", C.c_double * 3), ("scattering", C.c_double * 3), ("mean_cosine", C.c_double),
                ("continuation_prob", C.c_double)]


class Scene(C.Structure):
    _fields_ = [("n_media", C.c_int32), ("media", SceneMedium * SCENE_MAX_MEDIA), ("n_boxes", C.c_int32),
                ("box_lo", (C.c_double * 3) * MAX_BOXES), ("box_hi", (C.c_double * 3) * MAX_BOXES),
                ("box_medium", C.c_int32 * MAX_BOXES), ("camera_pos", C.c_double * 3), ("fov_deg", C.c_double),
                ("width", C.c_int32), ("height", C.c_int32), ("light_paths", C.c_int32),
                ("max_path_length", C.c_int32), ("light_size", C.c_double), ("light_intensity", C.c_double),
                ("techniques", C.c_uint32), ("query_beam_type", C.c_uint32), ("photon_beam_type", C.c_uint32),
                ("beam_length_cap", C.c_double), ("min_dist_to_med", C.c_double), ("bb1d_min_mfp", C.c_double),
                ("seed", C.c_uint64)]


def scene_struct(cfg) -> Scene:
    """upbp_scene of a :class:`smallupbp_b200.workload.SceneConfig` (the scene the host generator traces)."""
    from .workload import iteration_constants
    if len(cfg.boxes) > MAX_BOXES or len(cfg.media) > SCENE_MAX_MEDIA:
        raise ValueError("scene too large for upbp_scene")
    sc = Scene()
    sc.n_media = len(cfg.media)
    for i, m in enumerate(cfg.media):
        sc.media[i].absorption[:] = [float(x) for x in m.absorption]
        sc.media[i].scattering[:] = [float(x) for x in m.scattering]
        sc.media[i].mean_cosine = float(m.mean_cosine)
        sc.media[i].continuation_prob = float(m.continuation_prob)
    sc.n_boxes = len(cfg.boxes)
    for b, (lo, hi, mid) in enumerate(cfg.boxes):
        sc.box_lo[b][:] = [float(x) for x in lo]
        sc.box_hi[b][:] = [float(x) for x in hi]
        sc.box_medium[b] = mid
    sc.camera_pos[:] = [float(x) for x in cfg.camera_pos]
    sc.fov_deg = cfg.fov_deg
    sc.width, sc.height = cfg.width, cfg.height
    sc.light_paths = cfg.light_paths
    sc.max_path_length = cfg.max_path_length
    sc.light_size, sc.light_intensity = cfg.light_size, cfg.light_intensity
    sc.techniques, sc.query_beam_type, sc.photon_beam_type = cfg.techniques, cfg.query_beam_type, cfg.photon_beam_type
    sc.beam_length_cap = cfg.beam_length_cap
    sc.min_dist_to_med = cfg.min_dist_to_med
    sc.bb1d_min_mfp = iteration_constants(cfg)["bb1d_min_mfp"]
    sc.seed = cfg.seed
    return sc


assert C.sizeof(Mis) == 60
assert C.sizeof(Medium) == MEDIUM_DTYPE.itemsize
assert C.sizeof(Params) == PARAMS_DTYPE.itemsize

_PTR = {np.float32: f32p, np.int32: i32p, np.uint32: u32p, np.int64: i64p, np.uint64: u64p}


def ptr(a: np.ndarray, ctype=None):
    """Pointer to a C-contiguous numpy array (NULL for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    if ctype is None:
        ctype = _PTR[a.dtype.type]
    return a.ctypes.data_as(ctype)


def make_structs(w: Dict[str, np.ndarray]) -> Tuple[dict, List[np.ndarray]]:
    """Build the upbp_gpu.h structs for workload ``w``; returns (structs, keepalive)."""
    keep: List[np.ndarray] = []

    def a(name, dtype=None):
        """The array `name`, or None when the workload leaves it out (an MIS input of a workload
        without MIS, which the C ABI then receives as NULL)."""
        if name not in w:
            return None
        x = np.ascontiguousarray(w[name]) if dtype is None else np.ascontiguousarray(w[name], dtype=dtype)
        keep.append(x)
        return x

    def mis_ptr(x):
        return None if x is None else x.ctypes.data_as(C.POINTER(Mis))

    params = Params.from_buffer_copy(a("params").tobytes())
    media_arr = a("media")
    media = (Medium * len(media_arr)).from_buffer_copy(media_arr.tobytes())
    lv_ends = a("lv_path_ends")
    lv = LightVertices(
        n=len(w["lv_path_length"]), position=ptr(a("lv_position")), throughput=ptr(a("lv_throughput")),
        dir_fix=ptr(a("lv_dir_fix")), cont_prob=ptr(a("lv_cont_prob")), path_idx=ptr(a("lv_path_idx")),
        path_length=ptr(a("lv_path_length")), medium_id=ptr(a("lv_medium_id")), flags=ptr(a("lv_flags")),
        mis=mis_ptr(a("lv_mis")), n_paths=0 if lv_ends is None else len(lv_ends), path_ends=ptr(lv_ends))
    beams = Beams(
        n=len(w["beam_length"]), origin=ptr(a("beam_origin")), direction=ptr(a("beam_direction")),
        length=ptr(a("beam_length")), throughput=ptr(a("beam_throughput")), flags=ptr(a("beam_flags")),
        ray_sample_pdf=ptr(a("beam_ray_sample_pdf")), ray_sample_rev_pdf=ptr(a("beam_ray_sample_rev_pdf")),
        ray_sampling_flags=ptr(a("beam_ray_sampling_flags")), last_pdf_w_inv=ptr(a("beam_last_pdf_w_inv")),
        medium_id=ptr(a("beam_medium_id")), light_vertex=ptr(a("beam_light_vertex")))
    sq = SegmentQueries(
        n=len(w["sq_path_length"]), origin=ptr(a("sq_origin")), direction=ptr(a("sq_direction")),
        seg_begin=ptr(a("sq_seg_begin")), seg_count=ptr(a("sq_seg_count")), flags=ptr(a("sq_flags")),
        path_length=ptr(a("sq_path_length")), last_pdf_w_inv=ptr(a("sq_last_pdf_w_inv")),
        throughput=ptr(a("sq_throughput")), pixel=ptr(a("sq_pixel")), cam_mis_begin=ptr(a("sq_cam_mis_begin")),
        n_segments=len(w["seg_dist_min"]), seg_dist_min=ptr(a("seg_dist_min")), seg_dist_max=ptr(a("seg_dist_max")),
        seg_pdf=ptr(a("seg_pdf")), seg_rev_pdf=ptr(a("seg_rev_pdf")), seg_attenuation=ptr(a("seg_attenuation")),
        seg_medium=ptr(a("seg_medium")))
    pq = PointQueries(
        n=len(w["pq_path_length"]), position=ptr(a("pq_position")), dir_fix=ptr(a("pq_dir_fix")),
        medium_id=ptr(a("pq_medium_id")), path_length=ptr(a("pq_path_length")), throughput=ptr(a("pq_throughput")),
        pixel=ptr(a("pq_pixel")), cam_mis_begin=ptr(a("pq_cam_mis_begin")))
    cm = a("cam_mis")
    structs = dict(params=params, media=media, n_media=len(media_arr), lv=lv, beams=beams, sq=sq, pq=pq,
                   cam_mis=mis_ptr(cm), n_cam_mis=0 if cm is None else len(cm))
    return structs, keep
