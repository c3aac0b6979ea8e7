"""Host-side checks of the C ABI that need no GPU: the library loads, exports every entry point
declared in include/upbp_gpu.h, the ctypes mirror has the header's layout, and calls fail cleanly."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from smallupbp_b200 import abi, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "upbp_gpu.h")


def declared_entry_points():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(upbp_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(engine.LIB_PATH):
        from smallupbp_b200 import build
        build.build()
    return C.CDLL(engine.LIB_PATH)


def test_library_exports_every_declared_entry_point(lib):
    names = declared_entry_points()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(engine.EXPORTS) <= set(names)


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\nint main(void){printf("%%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu %%zu\\n",'
                   'sizeof(upbp_mis), sizeof(upbp_medium), sizeof(upbp_params), sizeof(upbp_light_vertices),'
                   'sizeof(upbp_beams), sizeof(upbp_segment_queries), sizeof(upbp_point_queries), sizeof(upbp_query_stats), sizeof(upbp_tuning),'
                   'sizeof(upbp_bb1d_grid));return 0;}' % HEADER)
    exe = tmp_path / "sizes"
    subprocess.check_call(["gcc", str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    want = [C.sizeof(t) for t in (abi.Mis, abi.Medium, abi.Params, abi.LightVertices, abi.Beams,
                                  abi.SegmentQueries, abi.PointQueries, abi.QueryStats, abi.Tuning, abi.Bb1dGrid)]
    assert got == want


def test_create_without_device_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    ctx = C.c_void_p()
    lib.upbp_ctx_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    assert lib.upbp_ctx_create(C.byref(ctx), 0) == -3  # UPBP_ERR_CUDA
    assert not ctx.value
    lib.upbp_ctx_destroy.argtypes = [C.c_void_p]
    assert lib.upbp_ctx_destroy(None) == -1  # UPBP_ERR_INVALID_ARG
    with pytest.raises(engine.UpbpError):
        engine.EstimatorStage(0)


def test_no_cpu_fallback_in_product_package():
    # The product path must not route through the oracle or any CPU estimator.
    pkg = os.path.join(ROOT, "smallupbp_b200")
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            text = open(os.path.join(pkg, f)).read()
            assert not re.search(r"^\s*(from|import)\s+oracle", text, re.M), f
            assert "liboracle" not in text and "libupbp_ref" not in text, f


def test_context_destroy_frees_every_device_buffer():
    # upbp_ctx_destroy frees the buffers it lists; every DBuf member of the context must be listed,
    # or its device memory outlives the context
    src = open(os.path.join(ROOT, "smallupbp_b200", "csrc", "upbp_capi.cu")).read()
    i = src.index("struct upbp_ctx")
    body = src[i:src.index("\n};\n", i)]
    members = set()
    for m in re.finditer(r"\bDBuf\s+([^;]+);", body):
        members.update(n.strip() for n in m.group(1).split(","))
    k = src.index("DBuf* all[] = {")
    freed = set(re.findall(r"&c->(\w+)", src[k:src.index("};", k)]))
    assert members and members <= freed, sorted(members - freed)
