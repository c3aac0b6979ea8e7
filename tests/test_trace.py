"""Device-side light and camera passes (upbp_trace_light_paths / upbp_trace_camera_paths).

The checker is the host generator (smallupbp_b200/workload.py): the same per-path Philox streams,
the same FP64 arithmetic in the same order.  Integer records (path indices, lengths, media, flags,
offsets, counts) must match exactly; floating-point records to within a few FP32 ulps, since
log/exp/sin/cos of CUDA and of numpy may differ in the last bit of a double.  A traced iteration
must then give the estimator stage the same candidates and image as the uploaded generator
iteration.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from smallupbp_b200 import abi, engine
from smallupbp_b200 import workload as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLOAT_RTOL = 1e-6  # ~8 FP32 ulps

CASES = {
    "cube_short": lambda: W.cube_scene("cube24x1536", 24, 24, 1536, 6, 0.02),
    "cube_long_capped": lambda: W.cube_scene("cube_long", 32, 32, 4096, 6, 0.01, photon_beam_type=W.LONG_BEAM,
                                             beam_length_cap=0.3),
    "boxes_nested": lambda: W.nested_boxes_scene("boxes_small", 32, 32, 4096, 6, 0.02),
    "short_queries_bb1d_previous": lambda: W.cube_scene(
        "cube_sq", 24, 24, 2048, 5, 0.02, query_beam_type=W.SHORT_BEAM,
        techniques=W.BPT | W.SURF | W.PP3D | W.PB2D | W.BB1D | W.BB1D_PREVIOUS, min_dist_to_med=0.1),
}


# ------------------------------------------------------------------ CPU: random numbers, layout

def test_philox_matches_numpys_bit_generator():
    """numpy's Philox (4x64-10) increments its counter before each block: counter c - 1 in numpy
    gives our block c."""
    rng = np.random.default_rng(5)
    for _ in range(20):
        ctr = [int(x) for x in rng.integers(1, 2 ** 63, 4, dtype=np.int64)]
        key = [int(x) for x in rng.integers(0, 2 ** 63, 2, dtype=np.int64)]
        ours = [int(x) for x in W.philox4x64([np.uint64(x) for x in ctr], key)]
        bg = np.random.Philox(counter=np.array([ctr[0] - 1] + ctr[1:], np.uint64), key=np.array(key, np.uint64))
        assert ours == [int(x) for x in bg.random_raw(4)]


def test_philox_known_answer():
    # Random123 known-answer vector for philox4x64_10: counter 0, key 0
    out = [int(x) for x in W.philox4x64([np.uint64(0)] * 4, (0, 0))]
    assert out == [0x16554D9ECA36314C, 0xDB20FE9D672D0FDC, 0xD7E772CEE186176B, 0x7E68B68AEC7BA23B]


def test_uniform_layout():
    key = (1234, 3)
    u = W.uniforms(key, W.LIGHT_STREAM, np.arange(5), 2, 0)
    assert u.shape == (5, 4) and (u >= 0).all() and (u < 1).all()
    f = W.flight_uniforms(key, W.LIGHT_STREAM, np.arange(5), 2, 6)
    np.testing.assert_array_equal(f[:, :4], W.uniforms(key, W.LIGHT_STREAM, np.arange(5), 2, 1))
    np.testing.assert_array_equal(f[:, 4:], W.uniforms(key, W.LIGHT_STREAM, np.arange(5), 2, 2)[:, :2])
    # a path's numbers do not depend on which other paths are drawn
    np.testing.assert_array_equal(W.uniforms(key, W.CAMERA_STREAM, np.array([3]), 1, 0)[0],
                                  W.uniforms(key, W.CAMERA_STREAM, np.arange(5), 1, 0)[3])


def test_scene_struct_layout_matches_the_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "upbp_gpu.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu\\n", sizeof(upbp_scene), '
                   'offsetof(upbp_scene, n_boxes), offsetof(upbp_scene, camera_pos), '
                   'offsetof(upbp_scene, techniques), offsetof(upbp_scene, seed)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    want = [C.sizeof(abi.Scene), abi.Scene.n_boxes.offset, abi.Scene.camera_pos.offset,
            abi.Scene.techniques.offset, abi.Scene.seed.offset]
    assert got == want


def test_scene_struct_of_a_config():
    cfg = W.config("boxes3")
    sc = abi.scene_struct(cfg)
    assert sc.n_boxes == 3 and sc.n_media == 4
    assert list(sc.box_lo[1]) == [0.2, 0.2, 0.2] and sc.box_medium[2] == 3
    assert sc.media[1].absorption[0] == cfg.media[1].absorption[0]  # FP64, not rounded to FP32


# ------------------------------------------------------------------ GPU: against the generator

def compare_inputs(got, want, names):
    for name in names:
        a, b = got[name], want[name]
        assert a.shape == b.shape, (name, a.shape, b.shape)
        if a.dtype.names:  # MIS records
            for f in a.dtype.names:
                compare_values(a[f], b[f], "%s.%s" % (name, f))
        else:
            compare_values(a, b, name)


def compare_values(a, b, what):
    if a.dtype.kind in "iu":
        np.testing.assert_array_equal(a, b, err_msg=what)
        return
    # almost every value is bit-identical (all of them on the B200 runs so far); the tolerance
    # only admits last-bit differences of the double-precision math functions
    assert a.size < 100 or np.mean(a == b) >= 0.999, (what, float(np.mean(a == b)))
    a64, b64 = a.astype(np.float64), b.astype(np.float64)
    assert np.array_equal(np.isfinite(a64), np.isfinite(b64)), what
    fin = np.isfinite(b64)
    scale = np.abs(b64[fin]).max() if fin.any() else 0.0
    bad = np.abs(a64[fin] - b64[fin]) > FLOAT_RTOL * np.abs(b64[fin]) + 1e-12 * scale
    assert not bad.any(), (what, int(bad.sum()), a64[fin][bad][:4], b64[fin][bad][:4])
    np.testing.assert_array_equal(a64[~fin], b64[~fin], err_msg=what)


LIGHT = [n for n in engine.INPUT_ARRAYS if n.startswith(("lv_", "beam_"))]
CAMERA = [n for n in engine.INPUT_ARRAYS if not n.startswith(("lv_", "beam_"))]


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("iteration", [0, 3])
def test_device_passes_match_the_generator(case, iteration):
    cfg = CASES[case]()
    want = W.generate(cfg, iteration)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        st.trace(cfg, iteration)
        got = st.read_inputs()
    assert len(got["lv_path_idx"]) > 100 and len(got["beam_length"]) > 100 and len(got["sq_pixel"]) > 100
    compare_inputs(got, want, LIGHT)
    compare_inputs(got, want, CAMERA)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "mixed"])
def test_traced_iteration_evaluates_like_the_uploaded_one(mode):
    import golden_io as G

    m = engine.MODE_PLAIN if mode == "plain" else engine.MODE_MIXED
    cfg = W.config("cube64x4096")
    w = W.generate(cfg, 1)
    with engine.EstimatorStage(0, m) as st:
        st.run(w)
        want_img, want_stats = st.image(), st.query_stats()
        want_seg = st.segment_results()
    with engine.EstimatorStage(0, m) as st:
        st.trace(cfg, 1)
        st.build()
        st.clear_image()
        st.evaluate()
        img, stats, seg = st.image(), st.query_stats(), st.segment_results()
    for k in want_stats:
        if k.startswith("count"):
            np.testing.assert_array_equal(stats[k], want_stats[k], err_msg=k)
    for a, b, what in zip(seg, want_seg, ("PB2D", "BB1D")):
        G.assert_close(a, b, what)
    assert G.image_rel_l2(img, want_img) < 1e-5


@pytest.mark.gpu
def test_device_passes_at_full_size():
    """cube512 (262,144 light paths, 512x512 pixels): every array as the generator's."""
    cfg = W.config("cube512")
    want = W.generate(cfg, 2)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        got = st.trace(cfg, 2).read_inputs()
    assert len(got["lv_path_idx"]) > 300_000 and len(got["sq_pixel"]) > 200_000
    compare_inputs(got, want, LIGHT + CAMERA)


@pytest.mark.gpu
@pytest.mark.parametrize("max_len", [1, 2])
def test_short_paths_match_the_generator(max_len):
    cfg = W.cube_scene("cube_short_paths", 16, 16, 1024, max_len, 0.02)
    want = W.generate(cfg, 0)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        got = st.trace(cfg, 0).read_inputs()
    compare_inputs(got, want, LIGHT + CAMERA)


@pytest.mark.gpu
def test_a_single_light_path():
    cfg = W.cube_scene("cube_one_path", 16, 16, 1, 6, 0.02)
    want = W.generate(cfg, 0)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        got = st.trace(cfg, 0).read_inputs()
        st.build()
        st.clear_image()
        st.evaluate()
    assert len(got["lv_position"]) >= 1
    compare_inputs(got, want, LIGHT + CAMERA)


@pytest.mark.gpu
def test_invalid_scenes_are_refused():
    cfg = W.config("cube16x512")
    media, params = W.stage_constants(cfg, 0)
    with engine.EstimatorStage(0, engine.MODE_MIXED) as st:
        l = engine.lib()
        sc = abi.scene_struct(cfg)
        with pytest.raises(engine.UpbpError):  # params first
            st._ck(l.upbp_trace_light_paths(st._ctx, C.byref(sc), 0))
        st.set_media(media)
        prm = abi.Params.from_buffer_copy(np.ascontiguousarray(params).tobytes())
        st._ck(l.upbp_set_params(st._ctx, C.byref(prm)))
        for field, value in (("n_boxes", 0), ("n_boxes", abi.MAX_BOXES + 1), ("max_path_length", 17),
                             ("width", cfg.width + 1), ("techniques", cfg.techniques ^ W.PP3D), ("fov_deg", 0.0)):
            bad = abi.scene_struct(cfg)
            setattr(bad, field, value)
            rc = l.upbp_trace_camera_paths(st._ctx, C.byref(bad), 0)
            assert rc == -1, (field, value, rc)
        bad = abi.scene_struct(cfg)
        bad.box_medium[0] = 7
        assert l.upbp_trace_light_paths(st._ctx, C.byref(bad), 0) == -1
        st._ck(l.upbp_trace_light_paths(st._ctx, C.byref(sc), 0))  # the context still works
