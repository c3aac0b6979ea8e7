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
