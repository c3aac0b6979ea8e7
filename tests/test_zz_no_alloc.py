"""The allocation-free PP3D entry point (upbp_pp3d_evaluate_noalloc).

Callers such as a renderer plug-in inside a host application that owns the GPU memory budget, or
code running during CUDA graph capture, cannot allocate device memory.  This entry point gives them
the PP3D estimator (hash-grid build + RangeQuery) with all scratch memory inside the library: the
caller passes device buffers for the inputs and outputs only.  The test calls it through the C ABI
and checks it against the context-based entry point (upbp_evaluate, plain mode) within the parity
tolerance, on two calls in a row (the second call reuses the scratch array the first one left).

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import abi, engine

UPBP_ERR_CAPACITY = -6


def _device_structs(w, torch):
    """upbp_gpu.h structs whose array pointers are device buffers owned by the caller (torch)."""
    keep = []

    def dev(name):
        a = np.ascontiguousarray(w[name])
        t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
        keep.append(t)
        return t.data_ptr()

    def p(name, ctype):
        return C.cast(C.c_void_p(dev(name)), ctype)

    lv = abi.LightVertices(
        n=len(w["lv_path_idx"]), position=p("lv_position", abi.f32p), throughput=p("lv_throughput", abi.f32p),
        dir_fix=p("lv_dir_fix", abi.f32p), cont_prob=p("lv_cont_prob", abi.f32p),
        path_idx=p("lv_path_idx", abi.i32p), path_length=p("lv_path_length", abi.i32p),
        medium_id=p("lv_medium_id", abi.i32p), flags=p("lv_flags", abi.u32p),
        mis=p("lv_mis", C.POINTER(abi.Mis)), n_paths=len(w["lv_path_ends"]), path_ends=p("lv_path_ends", abi.i32p))
    pq = abi.PointQueries(
        n=len(w["pq_path_length"]), position=p("pq_position", abi.f32p), dir_fix=p("pq_dir_fix", abi.f32p),
        medium_id=p("pq_medium_id", abi.i32p), path_length=p("pq_path_length", abi.i32p),
        throughput=p("pq_throughput", abi.f32p), pixel=p("pq_pixel", abi.i32p),
        cam_mis_begin=p("pq_cam_mis_begin", abi.i64p))
    cam = p("cam_mis", C.POINTER(abi.Mis))
    params = abi.Params.from_buffer_copy(np.ascontiguousarray(w["params"]).tobytes())
    media_arr = np.ascontiguousarray(w["media"])
    media = (abi.Medium * len(media_arr)).from_buffer_copy(media_arr.tobytes())
    return params, media, len(media_arr), lv, pq, cam, keep


def _noalloc_fn():
    l = engine.lib()
    f = l.upbp_pp3d_evaluate_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Medium), C.c_int32, C.POINTER(abi.LightVertices),
                  C.POINTER(abi.Mis), C.POINTER(abi.PointQueries), abi.f32p, C.c_void_p]
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("path", [G.FIXTURES[-1], G.FIXTURES[0]], ids=G.name)
def test_noalloc_pp3d_matches_context_entry_point_twice(path):
    import torch

    w, _ = G.load(path)
    with engine.EstimatorStage(0, engine.MODE_PLAIN) as st:
        st.run(w)
        want = st.point_results()
    params, media, n_media, lv, pq, cam, keep = _device_structs(w, torch)
    f = _noalloc_fn()
    out = torch.full((max(pq.n, 1) * 3,), float("nan"), dtype=torch.float32, device="cuda")
    outp = C.cast(C.c_void_p(out.data_ptr()), abi.f32p)
    for call in range(2):
        out.fill_(float("nan"))
        rc = f(C.byref(params), media, n_media, C.byref(lv), cam, C.byref(pq), outp, None)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        got = out[: pq.n * 3].cpu().numpy().reshape(-1, 3)
        assert np.isfinite(got).all()
        G.assert_close(got, want, "no-alloc PP3D, call %d" % call)
    del keep


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_scratch():
    w, _ = G.load(G.FIXTURES[0])
    s, keep = abi.make_structs(w)
    lv = s["lv"]
    lv.n = (1 << 17) + 1  # UPBP_NOALLOC_MAX_LIGHT_VERTICES + 1; rejected before any device access
    out = np.zeros(3, np.float32)
    rc = _noalloc_fn()(C.byref(s["params"]), s["media"], s["n_media"], C.byref(lv), s["cam_mis"], C.byref(s["pq"]),
                       abi.ptr(out), None)
    assert rc == UPBP_ERR_CAPACITY
