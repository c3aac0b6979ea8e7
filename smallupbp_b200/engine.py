"""Python binding of the C ABI (``include/upbp_gpu.h``) implemented by ``libupbp_b200.so``.

:class:`EstimatorStage` owns one device context and mirrors the reference's per-iteration estimator
calls in batched form::

    stage = EstimatorStage(device=0)
    stage.load(workload)          # media, params, light vertices, beams  (HashGrid/EmbreeBre/PhotonBeamsEvaluator build inputs)
    stage.build()                 # HashGrid::Build + EmbreeBre::build + PhotonBeamsEvaluator::build
    stage.set_queries(workload)   # the recorded evalBre / evalBeamBeamEstimate / HashGrid::Process calls
    stage.evaluate()              # all of them in one batch
    stage.segment_results()       # per-call Rgb returned by evalBre / evalBeamBeamEstimate
    stage.point_results()         # per-call RangeQuery contribution
    stage.image()                 # framebuffer with the normalised contributions splatted

There is no CPU fallback: a missing or unloadable library, or a machine without a CUDA device,
raises :class:`UpbpError`.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libupbp_b200.so")

MODE_PLAIN, MODE_MIXED, MODE_FP64 = 0, 1, 2

EXPORTS = (
    "upbp_ctx_create", "upbp_ctx_destroy", "upbp_last_error", "upbp_set_mode", "upbp_set_tuning", "upbp_get_tuning",
    "upbp_set_bb1d_grid", "upbp_set_stream", "upbp_set_media", "upbp_set_params", "upbp_set_light_vertices", "upbp_set_beams",
    "upbp_build", "upbp_set_camera_mis", "upbp_set_segment_queries", "upbp_set_point_queries", "upbp_evaluate",
    "upbp_read_segment_results", "upbp_read_point_results", "upbp_read_query_stats", "upbp_clear_image",
    "upbp_read_image", "upbp_last_launch_count", "upbp_last_timings", "upbp_destroy_structures",
    "upbp_read_tested_counts", "upbp_adjoint", "upbp_device_bytes", "upbp_capture_graph", "upbp_launch_graph",
    "upbp_read_bp2d_results", "upbp_trace_light_paths", "upbp_trace_camera_paths", "upbp_read_input",
)

# the record arrays of the C ABI: name -> (dtype, values per record); upbp_read_input reads them back
INPUT_ARRAYS = {
    "lv_position": ("<f4", 3), "lv_throughput": ("<f4", 3), "lv_dir_fix": ("<f4", 3), "lv_cont_prob": ("<f4", 0),
    "lv_path_idx": ("<i4", 0), "lv_path_length": ("<i4", 0), "lv_medium_id": ("<i4", 0), "lv_flags": ("<u4", 0),
    "lv_mis": (None, 0), "lv_path_ends": ("<i4", 0),
    "beam_origin": ("<f4", 3), "beam_direction": ("<f4", 3), "beam_length": ("<f4", 0),
    "beam_throughput": ("<f4", 3), "beam_flags": ("<u4", 0), "beam_ray_sample_pdf": ("<f4", 0),
    "beam_ray_sample_rev_pdf": ("<f4", 0), "beam_ray_sampling_flags": ("<u4", 0),
    "beam_last_pdf_w_inv": ("<f4", 0), "beam_medium_id": ("<i4", 0), "beam_light_vertex": ("<i4", 0),
    "cam_mis": (None, 0),
    "sq_origin": ("<f4", 3), "sq_direction": ("<f4", 3), "sq_seg_begin": ("<i4", 0), "sq_seg_count": ("<i4", 0),
    "sq_flags": ("<u4", 0), "sq_path_length": ("<i4", 0), "sq_last_pdf_w_inv": ("<f4", 0),
    "sq_throughput": ("<f4", 3), "sq_pixel": ("<i4", 0), "sq_cam_mis_begin": ("<i8", 0),
    "seg_dist_min": ("<f4", 0), "seg_dist_max": ("<f4", 0), "seg_pdf": ("<f4", 0), "seg_rev_pdf": ("<f4", 0),
    "seg_attenuation": ("<f4", 3), "seg_medium": ("<i4", 0),
    "pq_position": ("<f4", 3), "pq_dir_fix": ("<f4", 3), "pq_medium_id": ("<i4", 0), "pq_path_length": ("<i4", 0),
    "pq_throughput": ("<f4", 3), "pq_pixel": ("<i4", 0), "pq_cam_mis_begin": ("<i8", 0),
}


class UpbpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("upbp error %d: %s" % (code, msg))
        self.code = code


_lib = None


def lib():
    """Load libupbp_b200.so (raises if it is missing: the CUDA path is the only path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise UpbpError(-4, "%s not built (python -m smallupbp_b200.build)" % LIB_PATH)
        l = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        l.upbp_ctx_create.argtypes = [C.POINTER(vp), C.c_int]
        l.upbp_ctx_destroy.argtypes = [vp]
        l.upbp_last_error.argtypes = [vp]
        l.upbp_last_error.restype = C.c_char_p
        l.upbp_set_mode.argtypes = [vp, C.c_int]
        l.upbp_set_tuning.argtypes = [vp, C.POINTER(abi.Tuning)]
        l.upbp_get_tuning.argtypes = [vp, C.POINTER(abi.Tuning)]
        l.upbp_set_bb1d_grid.argtypes = [vp, C.POINTER(abi.Bb1dGrid)]
        l.upbp_set_stream.argtypes = [vp, vp]
        l.upbp_set_media.argtypes = [vp, C.POINTER(abi.Medium), C.c_int32]
        l.upbp_set_params.argtypes = [vp, C.POINTER(abi.Params)]
        l.upbp_set_light_vertices.argtypes = [vp, C.POINTER(abi.LightVertices)]
        l.upbp_set_beams.argtypes = [vp, C.POINTER(abi.Beams)]
        l.upbp_build.argtypes = [vp]
        l.upbp_set_camera_mis.argtypes = [vp, C.POINTER(abi.Mis), C.c_int64]
        l.upbp_set_segment_queries.argtypes = [vp, C.POINTER(abi.SegmentQueries)]
        l.upbp_set_point_queries.argtypes = [vp, C.POINTER(abi.PointQueries)]
        l.upbp_evaluate.argtypes = [vp]
        l.upbp_read_segment_results.argtypes = [vp, abi.f32p, abi.f32p]
        l.upbp_read_point_results.argtypes = [vp, abi.f32p]
        l.upbp_read_query_stats.argtypes = [vp, C.POINTER(abi.QueryStats)]
        l.upbp_clear_image.argtypes = [vp]
        l.upbp_read_image.argtypes = [vp, abi.f32p]
        l.upbp_last_launch_count.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        l.upbp_last_timings.argtypes = [vp] + [C.POINTER(C.c_float)] * 4
        l.upbp_destroy_structures.argtypes = [vp]
        l.upbp_read_tested_counts.argtypes = [vp, abi.u64p]
        l.upbp_adjoint.argtypes = [vp, abi.f32p, C.c_int32, C.POINTER(C.c_double)]
        l.upbp_device_bytes.argtypes = [vp, abi.u64p]
        l.upbp_capture_graph.argtypes = [vp]
        l.upbp_read_bp2d_results.argtypes = [vp, abi.f32p, abi.u32p, abi.u64p]
        l.upbp_launch_graph.argtypes = [vp]
        l.upbp_trace_light_paths.argtypes = [vp, C.POINTER(abi.Scene), C.c_uint32]
        l.upbp_trace_camera_paths.argtypes = [vp, C.POINTER(abi.Scene), C.c_uint32]
        l.upbp_read_input.argtypes = [vp, C.c_char_p, vp, C.c_int64, C.POINTER(C.c_int64)]
        for name in EXPORTS:
            if name != "upbp_last_error":
                getattr(l, name).restype = C.c_int
        _lib = l
    return _lib


class EstimatorStage:
    """One device context of the batched estimator stage."""

    def __init__(self, device: int = 0, mode: int = MODE_PLAIN):
        self._l = lib()
        self._ctx = C.c_void_p()
        rc = self._l.upbp_ctx_create(C.byref(self._ctx), device)
        if rc != 0:
            raise UpbpError(rc, "upbp_ctx_create(device=%d) failed (no usable CUDA device?)" % device)
        self._keep = []
        self._nq = 0
        self._np = 0
        self._npix = 0
        self.set_mode(mode)

    # -------------------------------------------------------------- plumbing
    def _ck(self, rc: int):
        if rc != 0:
            raise UpbpError(rc, self._l.upbp_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            self._l.upbp_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_mode(self, mode: int):
        self._ck(self._l.upbp_set_mode(self._ctx, mode))

    def set_tuning(self, **kw):
        """Update any of pb2d_leaf, bb1d_leaf, block_threads, beam_piece_radii, bb1d_kernel, pb2d_kernel,
        query_order."""
        t = self.get_tuning()
        for k, v in kw.items():
            if not hasattr(t, k):
                raise KeyError(k)
            setattr(t, k, v)
        self._ck(self._l.upbp_set_tuning(self._ctx, C.byref(t)))

    def set_bb1d_grid(self, grid_res: int, max_beams_in_cell: int = 0, reduction: int = 0, seed: int = 1234):
        """BB1D over the reference's uniform beam grid of resolution ``grid_res`` (0: the LBVH over
        beam pieces), optionally reduced to ``max_beams_in_cell`` beams per cell (PRESAMPLE)."""
        g = abi.Bb1dGrid(grid_res=grid_res, max_beams_in_cell=max_beams_in_cell, reduction=reduction, seed=seed)
        self._ck(self._l.upbp_set_bb1d_grid(self._ctx, C.byref(g)))

    def get_tuning(self) -> "abi.Tuning":
        t = abi.Tuning()
        self._ck(self._l.upbp_get_tuning(self._ctx, C.byref(t)))
        return t

    def set_stream(self, stream_ptr: int):
        self._ck(self._l.upbp_set_stream(self._ctx, C.c_void_p(stream_ptr)))

    # -------------------------------------------------------------- inputs
    def load(self, w: Dict[str, np.ndarray], structs=None):
        """Upload media, params, light vertices and beams of workload ``w``."""
        s, keep = structs if structs is not None else abi.make_structs(w)
        self._keep = [keep, s]
        self._ck(self._l.upbp_set_media(self._ctx, s["media"], s["n_media"]))
        self._ck(self._l.upbp_set_params(self._ctx, C.byref(s["params"])))
        self._ck(self._l.upbp_set_light_vertices(self._ctx, C.byref(s["lv"])))
        self._ck(self._l.upbp_set_beams(self._ctx, C.byref(s["beams"])))
        self._npix = s["params"].image_width * s["params"].image_height
        return s

    def build(self):
        self._ck(self._l.upbp_build(self._ctx))

    def set_queries(self, w: Dict[str, np.ndarray], structs=None):
        s, keep = structs if structs is not None else abi.make_structs(w)
        self._keep.append((keep, s))
        self._ck(self._l.upbp_set_camera_mis(self._ctx, s["cam_mis"], s["n_cam_mis"]))
        self._ck(self._l.upbp_set_segment_queries(self._ctx, C.byref(s["sq"])))
        self._ck(self._l.upbp_set_point_queries(self._ctx, C.byref(s["pq"])))
        self._nq = s["sq"].n
        self._np = s["pq"].n

    def trace(self, cfg, iteration: int = 0):
        """The light and camera passes of iteration ``iteration`` of scene ``cfg`` (a
        :class:`workload.SceneConfig`) on the device: sets the media and params as the host
        generator does, then traces the light sub-paths and the camera sub-paths into the context.
        Follow with :meth:`build`, :meth:`clear_image` and :meth:`evaluate`."""
        from . import workload as W
        media, params = W.stage_constants(cfg, iteration)
        self.set_media(media)
        prm = abi.Params.from_buffer_copy(np.ascontiguousarray(params).tobytes())
        self._params_keep = prm
        self._ck(self._l.upbp_set_params(self._ctx, C.byref(prm)))
        sc = abi.scene_struct(cfg)
        self._ck(self._l.upbp_trace_light_paths(self._ctx, C.byref(sc), iteration))
        self._ck(self._l.upbp_trace_camera_paths(self._ctx, C.byref(sc), iteration))
        self._npix = cfg.width * cfg.height
        self._nq = self.input_bytes("sq_pixel") // 4
        self._np = self.input_bytes("pq_pixel") // 4
        return self

    def input_bytes(self, name: str) -> int:
        n = C.c_int64()
        self._ck(self._l.upbp_read_input(self._ctx, name.encode(), None, 0, C.byref(n)))
        return n.value

    def grid_structure(self) -> Dict[str, np.ndarray]:
        """The beam grid of the last build (upbp_set_bb1d_grid) as the reference holds it: ``cells``
        (mCells), ``beams`` (mPointers as beam indices) and ``pdfs`` (mPdfs, empty without a
        reduction)."""
        out = {}
        for key, name, dt in (("cells", "bb1d_grid_cells", np.uint32), ("beams", "bb1d_grid_beams", np.int32),
                              ("pdfs", "bb1d_grid_pdfs", np.float32)):
            nbytes = self.input_bytes(name)
            a = np.zeros(nbytes // 4, dt)
            if nbytes:
                self._ck(self._l.upbp_read_input(self._ctx, name.encode(), C.c_void_p(a.ctypes.data), nbytes, None))
            out[key] = a
        return out

    def read_inputs(self, names=None) -> Dict[str, np.ndarray]:
        """Copy stored input arrays back (as the workload dict names and shapes them)."""
        from .workload import MIS_DTYPE
        out = {}
        for name in names or INPUT_ARRAYS:
            dt, width = INPUT_ARRAYS[name]
            dtype = MIS_DTYPE if dt is None else np.dtype(dt)
            nbytes = self.input_bytes(name)
            a = np.zeros(nbytes // dtype.itemsize, dtype)
            if nbytes:
                self._ck(self._l.upbp_read_input(self._ctx, name.encode(), C.c_void_p(a.ctypes.data), nbytes, None))
            out[name] = a.reshape(-1, width) if width else a
        return out

    def clear_image(self):
        self._ck(self._l.upbp_clear_image(self._ctx))

    def evaluate(self):
        self._ck(self._l.upbp_evaluate(self._ctx))

    # -------------------------------------------------------------- outputs
    def segment_results(self):
        pb2d = np.zeros((self._nq, 3), np.float32)
        bb1d = np.zeros((self._nq, 3), np.float32)
        self._ck(self._l.upbp_read_segment_results(self._ctx, abi.ptr(pb2d), abi.ptr(bb1d)))
        return pb2d, bb1d

    def point_results(self):
        pp3d = np.zeros((self._np, 3), np.float32)
        self._ck(self._l.upbp_read_point_results(self._ctx, abi.ptr(pp3d)))
        return pp3d

    def query_stats(self):
        out = {k: np.zeros(self._nq if "pp3d" not in k else self._np, np.uint32 if k.startswith("count") else np.uint64)
               for k in ("count_pb2d", "hash_pb2d", "count_bb1d", "hash_bb1d", "count_pp3d", "hash_pp3d")}
        st = abi.QueryStats(**{k: abi.ptr(v) for k, v in out.items()})
        self._ck(self._l.upbp_read_query_stats(self._ctx, C.byref(st)))
        return out

    def bp2d_results(self):
        """B-P2D per point query: (rgb [n][3], accepted count, candidate hash)."""
        rgb = np.zeros((self._np, 3), np.float32)
        cnt = np.zeros(self._np, np.uint32)
        h = np.zeros(self._np, np.uint64)
        self._ck(self._l.upbp_read_bp2d_results(self._ctx, abi.ptr(rgb), abi.ptr(cnt), abi.ptr(h)))
        return rgb, cnt, h

    def capture_graph(self):
        """Record clear + build + evaluate of the current inputs as a CUDA graph (after one build and
        evaluate of them)."""
        self._ck(self._l.upbp_capture_graph(self._ctx))

    def launch_graph(self):
        self._ck(self._l.upbp_launch_graph(self._ctx))

    def device_bytes(self) -> int:
        out = np.zeros(1, np.uint64)
        self._ck(self._l.upbp_device_bytes(self._ctx, abi.ptr(out)))
        return int(out[0])

    def pixels(self) -> int:
        return self._npix

    def set_media(self, media: np.ndarray):
        """Replace the media table (``workload.MEDIUM_DTYPE`` records); the structures stay built."""
        m = np.ascontiguousarray(media, dtype=abi.MEDIUM_DTYPE)
        arr = (abi.Medium * len(m)).from_buffer_copy(m.tobytes())
        self._media_keep = arr
        self._ck(self._l.upbp_set_media(self._ctx, arr, len(m)))

    def adjoint(self, grad_image_ptr: int, medium: int) -> np.ndarray:
        """dL/d(sigma_a rgb, sigma_s rgb, g) of ``medium`` given dL/d framebuffer at ``grad_image_ptr``
        ([H*W][3] float32, host or device address)."""
        out = (C.c_double * 7)()
        self._ck(self._l.upbp_adjoint(self._ctx, C.cast(C.c_void_p(grad_image_ptr), abi.f32p), medium, out))
        return np.array(list(out), np.float64)

    def tested_counts(self):
        """Candidates tested by the last evaluate: {"pb2d": photons, "bb1d": beam pieces, "pp3d": photons}."""
        out = np.zeros(3, np.uint64)
        self._ck(self._l.upbp_read_tested_counts(self._ctx, abi.ptr(out)))
        return {"pb2d": int(out[0]), "bb1d": int(out[1]), "pp3d": int(out[2])}

    def image(self):
        img = np.zeros((self._npix, 3), np.float32)
        self._ck(self._l.upbp_read_image(self._ctx, abi.ptr(img)))
        return img

    def read_image_into(self, ptr: int):
        """Copy the framebuffer (H*W*3 float32) to ``ptr`` (host or device address)."""
        self._ck(self._l.upbp_read_image(self._ctx, C.cast(C.c_void_p(ptr), abi.f32p)))

    def launch_counts(self):
        b, e = C.c_int(), C.c_int()
        self._ck(self._l.upbp_last_launch_count(self._ctx, C.byref(b), C.byref(e)))
        return b.value, e.value

    def timings(self):
        v = [C.c_float() for _ in range(4)]
        self._ck(self._l.upbp_last_timings(self._ctx, *[C.byref(x) for x in v]))
        return dict(build_ms=v[0].value, pp3d_ms=v[1].value, pb2d_ms=v[2].value, bb1d_ms=v[3].value)

    def run(self, w: Dict[str, np.ndarray]):
        """Convenience: load, build, set queries, clear the image and evaluate."""
        s = abi.make_structs(w)
        self.load(w, s)
        self.build()
        self.set_queries(w, s)
        self.clear_image()
        self.evaluate()
        return self
