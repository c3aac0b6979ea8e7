#!/usr/bin/env python3
"""Build the reference SmallUPBP estimator code into ``oracle/_ref/`` (test infrastructure).

This recipe compiles the reference's OWN estimator sources -- ``Bre/Bre.cxx``
(PB2D / BRE), ``Beams/PhBeams.cxx`` with ``PhBrute.hxx`` and ``PhGrid.hxx``
(BB1D), ``Misc/HashGrid.hxx`` (PP3D), ``Path/PathWeight.hxx`` (UPBP MIS),
``Path/PhaseFunction.hxx`` and ``Scene/Media.hxx`` -- together with the
harness ``oracle/ref_harness.cpp`` into one shared library,
``oracle/_ref/libupbp_ref.so``.  The harness reads the repository's neutral
SoA workload (the same arrays the CUDA path consumes) and calls the reference
functions on it, so the reference itself produces the golden outputs.

The reference is MSVC 2013 code; g++ needs a handful of mechanical source
fixes (backslash include paths, ``__declspec(align)``, missing ``typename``,
MSVC-only casts).  They are applied to a COPY under ``oracle/_ref/src`` (which
is git-ignored and never committed); the reference tree is only read.

Embree 2.0 is built too: its 40 core, BVH and ``sys`` sources (``EMBREE_SOURCES``)
are compiled from the same patched copy and linked in, so ``EmbreeBre`` runs on
Embree's own BVH and callback interface, exactly as the reference renderer does.

Usage: python oracle/build_ref.py [--reference DIR]
(DIR defaults to $UPBP_REFERENCE_DIR, else /root/reference.)
Exit status 0 and prints the built path; exits 2 (with a message) when the
reference tree is absent (e.g. on a machine that only runs prebuilt files).
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")

# Directories copied from the reference (headers and the two estimator .cxx files).
COPY_DIRS = [
    ("SmallUPBP/src", (".hxx", ".cxx", ".h")),
    ("embree-2.0/embree", (".h", ".cpp")),
    ("OpenEXR", (".h",)),
]

CASE_FIXES = {
    "Debugimages.hxx": "DebugImages.hxx",
    "Beamdensity.hxx": "BeamDensity.hxx",
}


def reference_dir() -> str:
    """Where the reference checkout lives: $UPBP_REFERENCE_DIR, else the default checkout path."""
    return os.environ.get("UPBP_REFERENCE_DIR", "/root/reference")


def copy_tree(ref: str) -> None:
    if os.path.isdir(SRC):
        shutil.rmtree(SRC)
    for rel, exts in COPY_DIRS:
        src_dir = os.path.join(ref, rel)
        for root, _dirs, files in os.walk(src_dir):
            # OpenEXR: only the top-level public headers are needed.
            if rel == "OpenEXR" and root != src_dir:
                continue
            for f in files:
                if not f.endswith(exts):
                    continue
                s = os.path.join(root, f)
                d = os.path.join(SRC, os.path.relpath(s, ref))
                os.makedirs(os.path.dirname(d), exist_ok=True)
                shutil.copyfile(s, d)


def patch_text(path: str, text: str) -> str:
    rel = os.path.relpath(path, SRC).replace(os.sep, "/")

    def fix_include(m: re.Match) -> str:
        inc = m.group(1).replace("\\", "/")
        for bad, good in CASE_FIXES.items():
            inc = inc.replace(bad, good)
        return '#include "%s"' % inc

    text = re.sub(r'#include\s+"([^"]+)"', fix_include, text)
    text = re.sub(r"__declspec\s*\(\s*align\s*\(\s*(\d+)\s*\)\s*\)", r"__attribute__((aligned(\1)))", text)
    text = text.replace("std::sqrtf(", "sqrtf(")

    if rel.endswith("Misc/Timer.hxx"):
        text = text.replace("#include <winsock2.h>", '#include "win_timer_shim.h"')
        text = text.replace("#include <windows.h>", "")
    if rel.endswith("PrecompiledLibs/FastFloat/FastFloat.h"):
        # (float&)__m128 reinterpretation -> lane-0 extract
        text = re.sub(r"\(float\s*&\)([^;]*);", r"_mm_cvtss_f32(\1);", text)
    if rel.endswith("Misc/Defs.hxx"):
        # embree's sys/platform.h already declares int8/uint8 ... with the g++ spellings
        text = re.sub(r"typedef\s+(unsigned\s+)?__int(8|16|64)\s+u?int(8|16|64)\s*;", "", text)
    if rel.endswith("Path/PriorityStack.hxx"):
        text = re.sub(r"(?<!typename )(std::forward_list<std::pair<ElementType, int>>\s*::const_iterator)",
                      r"typename \1", text)
    if rel.endswith("Scene/Scene.hxx"):
        text = text.replace("return Intersect(Ray(aPoint, aDir), Isect(aTMax),",
                            "Isect isectTmp(aTMax); return Intersect(Ray(aPoint, aDir), isectTmp,")
    if rel.endswith("Misc/Framebuffer.hxx"):
        text = text.replace("void Save(std::string & aFilename", "void Save(const std::string & aFilename")
    if rel.endswith("Structs/BoundingBox.hxx"):
        text = text.replace("BoundingBox3 result;", "BoundingBox result;")
        text = re.sub(r"(?<!typename )(?<!Pos::)\bTPoint::DirType(?!::)", "typename TPoint::DirType", text)
        text = re.sub(r"^(?:INLINE\s+)?([\w:<>]+)\s+(BoundingBox3|BoundingBox<Pos>)::",
                      r"template<> inline \1 \2::", text, flags=re.M)
    if rel.endswith("Beams/PhBeams.hxx"):
        # config switch so the harness can build the reference's brute-force AccelStruct too
        text = text.replace("#define USE_GRID",
                            "#if defined(UPBP_REF_USE_BRUTE)\n#define USE_BRUTE\n#else\n#define USE_GRID\n#endif")
    if rel.endswith("embree-2.0/embree/simd/sseb.h"):
        text = re.sub(
            r"_mm_shuffle_epi32\(\s*a\s*,\s*_MM_SHUFFLE\(([^)]*)\)\s*\)",
            r"_mm_castsi128_ps(_mm_shuffle_epi32(_mm_castps_si128(a), _MM_SHUFFLE(\1)))",
            text,
        )
    if rel.endswith("embree-2.0/embree/sys/intrinsics.h"):
        text = re.sub(r"\b__rdtsc\b", "embree_rdtsc", text)
        text = re.sub(r"\b__rdpmc\b", "embree_rdpmc", text)
    return text


def patch_tree() -> None:
    for root, _dirs, files in os.walk(SRC):
        for f in files:
            p = os.path.join(root, f)
            with open(p, "r", encoding="latin-1") as fh:
                t = fh.read()
            t2 = patch_text(p, t)
            if t2 != t:
                with open(p, "w", encoding="latin-1") as fh:
                    fh.write(t2)
    # Small generated shims (our own files, written into the copy).
    sysdir = os.path.join(SRC, "embree-2.0/embree/sys")
    with open(os.path.join(sysdir, "CMakeDefines.h"), "w") as fh:
        fh.write('#define CMAKE_SHARED_LIBRARY_PREFIX "lib"\n#define CMAKE_SHARED_LIBRARY_SUFFIX ".so"\n#define CMAKE_BUILD_DIR "."\n')
    with open(os.path.join(SRC, "SmallUPBP/src/Misc/win_timer_shim.h"), "w") as fh:
        fh.write(
            "#pragma once\n#include <chrono>\n#include <cstdint>\n"
            "typedef union { long long QuadPart; } LARGE_INTEGER;\n"
            "inline int QueryPerformanceCounter(LARGE_INTEGER* c){ c->QuadPart = (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count(); return 1; }\n"
            "inline int QueryPerformanceFrequency(LARGE_INTEGER* f){ f->QuadPart = 1000000000LL; return 1; }\n"
        )


EMBREE_SOURCES = """
embree.cpp common/alloc.cpp common/stat.cpp common/accel.cpp common/registry_accel.cpp
common/registry_builder.cpp common/registry_intersector.cpp geometry/triangle_mesh.cpp
geometry/virtual_scene.cpp builders/primrefgen.cpp builders/heuristic_binning.cpp
builders/heuristic_spatial.cpp builders/splitter.cpp builders/splitter_parallel.cpp
builders/splitter_fallback.cpp bvh2/bvh2.cpp bvh2/bvh2_intersector1.cpp bvh2/bvh2_intersector4.cpp
bvh4/bvh4.cpp bvh4/bvh4_intersector1.cpp bvh4/bvh4_intersector4_single.cpp
bvh4/bvh4_intersector4_chunk.cpp bvh4/bvh4_intersector4_hybrid.cpp bvh4i/bvh4i.cpp
bvh4i/bvh4i_intersector1.cpp bvh4mb/bvh4mb.cpp bvh4mb/bvh4mb_builder.cpp
bvh4mb/bvh4mb_intersector1.cpp bvh4mb/bvh4mb_intersector4.cpp sys/platform.cpp sys/sysinfo.cpp
sys/filename.cpp sys/library.cpp sys/thread.cpp sys/network.cpp sys/taskscheduler.cpp
sys/taskscheduler_sys.cpp sys/sync/mutex.cpp sys/sync/condition.cpp sys/stl/string.cpp
""".split()

CXX = ["g++", "-std=c++14", "-O2", "-msse4.2", "-fPIC", "-w", "-fpermissive"]


def _run_all(jobs: list[list[str]], cwd: str | None = None) -> None:
    """Run compile jobs, at most os.cpu_count() at a time; raise on the first failure."""
    procs: list[tuple[subprocess.Popen, list[str]]] = []
    limit = max(1, os.cpu_count() or 1)
    pending = list(jobs)
    failed = None
    while pending or procs:
        while pending and len(procs) < limit:
            cmd = pending.pop(0)
            procs.append((subprocess.Popen(cmd, cwd=cwd), cmd))
        p, cmd = procs.pop(0)
        if p.wait() != 0 and failed is None:
            failed = cmd
    if failed:
        raise RuntimeError("compile failed: " + " ".join(failed))


def compile_lib() -> str:
    obj = os.path.join(OUT, "obj")
    os.makedirs(obj, exist_ok=True)
    emb = os.path.join(SRC, "embree-2.0/embree")
    jobs, objs = [], []
    for s in EMBREE_SOURCES:
        o = os.path.join(obj, "embree_" + s.replace("/", "_") + ".o")
        objs.append(o)
        jobs.append(CXX + ["-D__SSE4_1__", "-I", emb, "-I", os.path.join(emb, "sys"), "-c", os.path.join(emb, s), "-o", o])
    inc = ["-fopenmp", "-include", os.path.join(HERE, "ref_compat.h"), "-I", os.path.join(SRC, "SmallUPBP/src"),
           "-I", emb, "-I", os.path.join(SRC, "OpenEXR"), "-I", HERE]
    for name, src, extra in (("harness", "ref_harness.cpp", []), ("bre", "ref_bre.cpp", []),
                             ("beams_grid", "ref_beams.cpp", []),
                             ("beams_brute", "ref_beams.cpp", ["-DUPBP_REF_USE_BRUTE"])):
        o = os.path.join(obj, name + ".o")
        objs.append(o)
        jobs.append(CXX + inc + extra + ["-c", os.path.join(HERE, src), "-o", o])
    _run_all(jobs)
    out_so = os.path.join(OUT, "libupbp_ref.so")
    subprocess.check_call(CXX + ["-shared", "-fopenmp", "-o", out_so] + objs + ["-lpthread", "-ldl"])
    return out_so


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_dir())
    ap.add_argument("--no-copy", action="store_true", help="reuse the patched copy")
    args = ap.parse_args()
    if not os.path.isdir(os.path.join(args.reference, "SmallUPBP/src")):
        print("reference tree not found at %s; oracle/_ref not built" % args.reference)
        return 2
    os.makedirs(OUT, exist_ok=True)
    if not args.no_copy:
        copy_tree(args.reference)
        patch_tree()
    print(compile_lib())
    return 0


if __name__ == "__main__":
    sys.exit(main())
