"""The allocation-free PP3D entry point (upbp_pp3d_evaluate_noalloc).

Some callers cannot allocate device memory: a renderer plug-in inside a host application that owns
the GPU memory budget and forbids plug-ins to allocate, or an embedded caller that reserves all
device memory up front.  This entry point gives them the PP3D estimator (hash-grid build +
RangeQuery) with all scratch memory inside the library: the caller passes device buffers for the
inputs and outputs only.  The tests call it through the C ABI and check it against the
context-based entry point (upbp_evaluate, plain mode) and the reference's own PP3D outputs stored
in the fixtures, within the parity tolerance, on two calls in a row (the second call reuses the
scratch array the first one left); and on the edge cases of its scratch: no light vertices, no
light vertex in a medium, the largest hash grid and nearly the largest light-vertex count.

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import golden_io as G
from smallupbp_b200 import abi, engine
from smallupbp_b200 import workload as W

UPBP_ERR_CAPACITY = -6
UPBP_ERR_INVALID_ARG = -1
MAX_LV = MAX_CELLS = 1 << 17  # UPBP_NOALLOC_MAX_LIGHT_VERTICES, UPBP_NOALLOC_MAX_HASH_CELLS


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


def _context_pp3d(w):
    with engine.EstimatorStage(0, engine.MODE_PLAIN) as st:
        st.run(w)
        return st.point_results()


def _noalloc_twice(w, torch, n_lv=None):
    """Two calls in a row through the C ABI; returns both outputs."""
    params, media, n_media, lv, pq, cam, keep = _device_structs(w, torch)
    if n_lv is not None:
        lv.n = n_lv
    f = _noalloc_fn()
    out = torch.full((max(pq.n, 1) * 3,), float("nan"), dtype=torch.float32, device="cuda")
    outp = C.cast(C.c_void_p(out.data_ptr()), abi.f32p)
    res = []
    for call in range(2):
        out.fill_(float("nan"))
        rc = f(C.byref(params), media, n_media, C.byref(lv), cam, C.byref(pq), outp, None)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        got = out[: pq.n * 3].cpu().numpy().reshape(-1, 3)
        assert np.isfinite(got).all(), call
        res.append(got)
    del keep
    return res


FIXTURE_CASES = [p for p in G.FIXTURES if G.name(p) in ("boxes_all", "config0_cube128", "cube_wide_radius")]


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURE_CASES, ids=G.name)
def test_noalloc_pp3d_matches_context_entry_point_and_reference_twice(path):
    import torch

    w, r = G.load(path)
    want = _context_pp3d(w)
    for call, got in enumerate(_noalloc_twice(w, torch)):
        G.assert_close(got, want, "no-alloc PP3D vs upbp_evaluate, call %d" % call)
        G.assert_close(got, r["pp3d"], "no-alloc PP3D vs the reference, call %d" % call)


@pytest.mark.gpu
def test_noalloc_edge_cases_of_its_scratch():
    import torch

    w, _ = G.load(next(p for p in G.FIXTURES if G.name(p) == "cube_wide_radius"))
    assert w["pq_path_length"].size > 0
    # no light vertices at all: every PP3D contribution is zero (after a call that left photons in
    # the scratch array)
    _noalloc_twice(w, torch)
    for got in _noalloc_twice(w, torch, n_lv=0):
        assert not got.any()
    # light vertices, but none in a medium: no photons, the hash grid stays empty
    w2 = dict(w)
    w2["lv_flags"] = (w["lv_flags"] & ~np.uint32(W.LV_IN_MEDIUM)).astype(w["lv_flags"].dtype)
    want = _context_pp3d(w2)
    assert not want.any()
    for got in _noalloc_twice(w2, torch):
        assert not got.any()
    # the largest hash grid the scratch holds
    w3 = dict(w)
    w3["params"] = w["params"].copy()
    w3["params"]["hash_cells"] = MAX_CELLS
    want = _context_pp3d(w3)
    assert want.any()
    for call, got in enumerate(_noalloc_twice(w3, torch)):
        G.assert_close(got, want, "no-alloc PP3D, %d hash cells, call %d" % (MAX_CELLS, call))


@pytest.mark.gpu
def test_noalloc_near_the_light_vertex_limit():
    import torch

    w = W.generate(W.config("cube64x87000"), 0)
    n = len(w["lv_path_idx"])
    assert MAX_LV // 2 < n <= MAX_LV, n
    want = _context_pp3d(w)
    assert want.any()
    for call, got in enumerate(_noalloc_twice(w, torch)):
        G.assert_close(got, want, "no-alloc PP3D, %d light vertices, call %d" % (n, call))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    w, _ = G.load(G.FIXTURES[0])
    s, keep = abi.make_structs(w)
    lv = s["lv"]
    lv.n = (1 << 17) + 1  # UPBP_NOALLOC_MAX_LIGHT_VERTICES + 1; rejected before any device access
    out = np.zeros(3, np.float32)
    rc = _noalloc_fn()(C.byref(s["params"]), s["media"], s["n_media"], C.byref(lv), s["cam_mis"], C.byref(s["pq"]),
                       abi.ptr(out), None)
    assert rc == UPBP_ERR_CAPACITY


def test_noalloc_rejects_null_arrays_before_any_device_access():
    w, _ = G.load(G.FIXTURES[0])
    s, keep = abi.make_structs(w)
    out = np.zeros(3 * max(s["pq"].n, 1), np.float32)
    f = _noalloc_fn()
    lv = s["lv"]
    lv.mis = None
    assert f(C.byref(s["params"]), s["media"], s["n_media"], C.byref(lv), s["cam_mis"], C.byref(s["pq"]),
             abi.ptr(out), None) == UPBP_ERR_INVALID_ARG
    s, keep = abi.make_structs(w)
    assert f(C.byref(s["params"]), s["media"], s["n_media"], C.byref(s["lv"]), None, C.byref(s["pq"]),
             abi.ptr(out), None) == UPBP_ERR_INVALID_ARG
    pq = s["pq"]
    pq.position = None
    assert f(C.byref(s["params"]), s["media"], s["n_media"], C.byref(s["lv"]), s["cam_mis"], C.byref(pq),
             abi.ptr(out), None) == UPBP_ERR_INVALID_ARG
    del keep
