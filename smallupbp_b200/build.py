"""Build the CUDA library ``libupbp_b200.so`` in-tree for sm_100a (B200).

``python -m smallupbp_b200.build`` (or ``__graft_entry__.build()``) compiles every ``.cu`` file of
``smallupbp_b200/csrc`` with nvcc into one shared library next to this file.  nvcc cross-compiles
without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libupbp_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


# Per-file flags: the device-side light and camera passes reproduce the host generator's FP64
# operation order, so no multiply-add may be contracted there.
# upbp_trace.cu: the light and camera passes reproduce the host generator's FP64 arithmetic bit for
# bit, so no FMA contraction.  upbp_gather.cu: the contributions use the fast approximate FP32
# division (at most 2 ulp); the candidate predicates and the traversal use explicit IEEE
# intrinsics (__fdiv_rn, __frcp_rn, __fmul_rn, ...), which the flag does not change.
FILE_FLAGS = {"upbp_trace.cu": ["-fmad=false"], "upbp_gather.cu": ["-prec-div=false"]}


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(verbose: bool = False, extra=()) -> str:
    objs = []
    procs = []
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + FILE_FLAGS.get(os.path.basename(src), []) + list(extra) + [
            "-I", CSRC, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    for p, cmd in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
