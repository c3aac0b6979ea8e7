"""The C++ mirror of the reference's estimator interface (include/upbp_gpu.hpp) compiles against the
C ABI and links the library; without a GPU, creating a batch raises upbp_gpu::Error."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "smallupbp_b200")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_mirror_compiles_links_and_reports_errors(tmp_path):
    import torch

    exe = str(tmp_path / "mirror_smoke")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "mirror_smoke.cpp"), "-L", LIBDIR, "-lupbp_b200",
                           "-Wl,-rpath," + LIBDIR, "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    if torch.cuda.is_available():
        assert r.returncode == 0, r.stdout + r.stderr
    else:
        assert r.returncode == 3, r.stdout + r.stderr
        assert r.stdout.startswith("error ")


def _build_replay(tmp_path):
    so = str(tmp_path / "libbatch_replay.so")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "batch_replay.cpp"), "-L", LIBDIR, "-lupbp_b200",
                           "-Wl,-rpath," + LIBDIR, "-o", so])
    return so


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_batch_replay_builds_and_links(tmp_path):
    import ctypes

    lib = ctypes.CDLL(_build_replay(tmp_path))
    assert hasattr(lib, "replay_through_batch")


@pytest.mark.gpu
@pytest.mark.parametrize("fixture", ["cube_long_short", "boxes_all", "config0_cube128", "cube_nomis_long"])
def test_cpp_batch_drop_in_matches_reference(tmp_path, fixture):
    # The C++ drop-in (upbp_gpu::Batch) driven one recorded call at a time, as the binding in
    # UPBP::RunIteration drives it, reproduces the reference's per-call results and image.
    import ctypes as C

    import numpy as np

    import golden_io as G
    from smallupbp_b200 import abi

    lib = C.CDLL(_build_replay(tmp_path))
    f = lib.replay_through_batch
    f.restype = C.c_int
    w, r = G.load(next(p for p in G.FIXTURES if G.name(p) == fixture))
    s, keep = abi.make_structs(w)
    nq, npq = s["sq"].n, s["pq"].n
    npix = s["params"].image_width * s["params"].image_height
    img = np.zeros((npix, 3), np.float32)
    pb2d, bb1d, pp3d = (np.zeros((nq, 3), np.float32), np.zeros((nq, 3), np.float32),
                        np.zeros((max(npq, 1), 3), np.float32))
    err = C.create_string_buffer(512)
    rc = f(0, C.byref(s["params"]), s["media"], s["n_media"], C.byref(s["lv"]), C.byref(s["beams"]), s["cam_mis"],
           C.byref(s["sq"]), C.byref(s["pq"]), abi.ptr(img), abi.ptr(pb2d), abi.ptr(bb1d), abi.ptr(pp3d), err, 512)
    assert rc == 0, err.value.decode()
    G.assert_close(pb2d, r["pb2d"], "PB2D through Batch")
    G.assert_close(bb1d, r["bb1d_brute"], "BB1D through Batch")
    G.assert_close(pp3d[:npq], r["pp3d"], "PP3D through Batch")
    assert G.image_rel_l2(img, r["image"]) <= 1e-4
    del keep
