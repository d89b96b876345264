"""The C ABI library without a GPU: it loads, exports every declared symbol,
and its host-side validation returns the documented status codes."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REF, ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "ccs_cuda.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ccs_\w+_cuda)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from halfedgecatmullclark_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        from halfedgecatmullclark_b200 import build
        build.build()
    return _native.lib()


def test_every_declared_symbol_is_exported(lib):
    from halfedgecatmullclark_b200 import _native
    syms = declared_symbols()
    assert len(syms) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ccs_\w+_cuda)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    assert set(syms) == set(_native.SIGNATURES), set(syms) ^ set(_native.SIGNATURES)
    for s in syms:
        getattr(lib, s)


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "ccs_cuda.h"\nint main(void){ cc_Subd *s = ccs_Create_cuda(0, 1);\n'
                   ' ccs_Refine_Scatter_cuda(s); ccs_Release_cuda(s); return 0; }\n')
    for cc, std in (("gcc", "-std=c11"), ("g++", "-std=c++17")):
        r = subprocess.run([cc, std, "-fsyntax-only", "-I" + os.path.dirname(HEADER), "-x",
                            "c" if cc == "gcc" else "c++", str(src)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_header_shares_types_with_reference_header(tmp_path):
    ref = os.path.join(REF, "CatmullClark.h")
    if not os.path.exists(ref):
        pytest.skip("reference header not available")
    src = tmp_path / "t.c"
    src.write_text('#include "CatmullClark.h"\n#include "ccs_cuda.h"\n'
                   '_Static_assert(sizeof(cc_Halfedge_SemiRegular) == 16, "record");\n'
                   '_Static_assert(sizeof(cc_Crease) == 12, "crease");\n'
                   'int f(cc_Subd *s){ return ccs_Refine_Scatter_cuda(s) + ccs_HalfedgeTwinID(s, 0, 1); }\n')
    r = subprocess.run(["gcc", "-std=gnu11", "-fsyntax-only", "-I" + REF,
                        "-I" + os.path.dirname(HEADER), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_compat_header_keeps_the_reference_calls(tmp_path):
    """include/ccs_cuda_compat.h after CatmullClark.h: the reference's own
    calls, a call through a function pointer and an accessor compile."""
    ref = os.path.join(REF, "CatmullClark.h")
    if not os.path.exists(ref):
        pytest.skip("reference header not available")
    src = tmp_path / "t.c"
    src.write_text('#define CC_IMPLEMENTATION\n#include "CatmullClark.h"\n#include "ccs_cuda_compat.h"\n'
                   'static void Bench(void (*f)(cc_Subd *), cc_Subd *s) { f(s); }\n'
                   'int main(void) { cc_Mesh *m = ccm_Load("x.ccm"); cc_Subd *s = ccs_Create(m, 2);\n'
                   '  ccs_Refine_Scatter(s); Bench(&ccs_Refine_Gather, s);\n'
                   '  cc_VertexPoint p = ccs_VertexPoint(s, 0, 2); (void)p;\n'
                   '  ccs_Release(s); ccm_Release(m); return 0; }\n')
    for cc, std in (("gcc", "-std=gnu11"), ("g++", "-std=c++17")):
        r = subprocess.run([cc, std, "-fsyntax-only", "-I" + REF, "-I" + os.path.dirname(HEADER),
                            "-x", "c" if cc == "gcc" else "c++", str(src)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_compat_header_maps_every_subd_call():
    """Every subd call the reference declares (ccs_Create, ccs_Release,
    ccs_Refine*) has a same-named macro in include/ccs_cuda_compat.h, and each
    maps to a `_cuda` entry point the library exports."""
    ref = os.path.join(REF, "CatmullClark.h")
    if not os.path.exists(ref):
        pytest.skip("reference header not available")
    with open(ref) as fh:
        decl = set(re.findall(r"^CCDEF [^(]*?\b(ccs_(?:Create|Release|Refine\w*))\(", fh.read(), re.M))
    compat = os.path.join(os.path.dirname(HEADER), "ccs_cuda_compat.h")
    with open(compat) as fh:
        text = fh.read()
    mapped = set(re.findall(r"^#define (ccs_\w+)\s+ccs_compat_\w+", text, re.M))
    assert decl and decl <= mapped, decl - mapped
    from halfedgecatmullclark_b200 import _native
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    for name in decl:
        assert re.search(r"\b%s_cuda\b" % name, out), name


def test_error_strings(lib):
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert lib.ccs_ErrorString_cuda(code)
    assert b"sm_100a" in lib.ccs_Version_cuda()


def test_invalid_arguments_are_refused_on_the_host(lib):
    from halfedgecatmullclark_b200 import configs
    out = ctypes.c_void_p()
    assert lib.ccs_CreateEx_cuda(None, 3, 0, ctypes.byref(out)) == -1
    assert lib.ccs_LastError_cuda() == -1
    w = configs.torus_quads()
    m = w.cage.as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(m), 0, 0, ctypes.byref(out)) == -1     # depth 0
    assert lib.ccs_CreateEx_cuda(ctypes.byref(m), 3, 0, None) == -1                 # no out
    bad = w.cage.copy()
    bad.halfedges["twinID"][5] = bad.H + 3                                          # twin out of range
    mb = bad.as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(mb), 3, 0, ctypes.byref(out)) == -1
    bad = w.cage.copy()
    bad.halfedges["nextID"][0], bad.halfedges["nextID"][1] = bad.halfedges["nextID"][1], bad.halfedges["nextID"][0]
    mb = bad.as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(mb), 3, 0, ctypes.byref(out)) == -1   # next/prev broken
    bad = w.cage.copy()
    bad.creases["nextID"][2] = -5
    mb = bad.as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(mb), 3, 0, ctypes.byref(out)) == -1   # crease link
    # an isolated vertex (no halfedge: the reference's gather rules would
    # follow its vertex-to-halfedge entry of -1)
    from halfedgecatmullclark_b200.cage import build_cage
    pts = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [2, 2, 2]], np.float32)
    iso = build_cage(pts, [[0, 1, 2, 3]]).as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(iso), 2, 0, ctypes.byref(out)) == -1
    big = configs.height_grid(n=256)
    mg = big.cage.as_cc_mesh()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(mg), 6, 0, ctypes.byref(out)) == -3   # int32 overflow
    # calls on a subd this library did not create
    fake = ctypes.create_string_buffer(64)
    assert lib.ccs_Refine_Scatter_cuda(fake) == -1
    assert lib.ccs_Download_cuda(fake) == -1
    lib.ccs_Release_cuda(None)


def test_create_without_gpu_reports_cuda_error(lib):
    if gpu_available():
        pytest.skip("a GPU is present")
    from halfedgecatmullclark_b200 import configs
    w = configs.torus_quads()
    m = w.cage.as_cc_mesh()
    out = ctypes.c_void_p()
    assert lib.ccs_CreateEx_cuda(ctypes.byref(m), 2, 0, ctypes.byref(out)) == -4
    assert not out.value


def test_build_cage_without_gpu_reports_an_error(lib):
    if gpu_available():
        pytest.skip("a GPU is present")
    from halfedgecatmullclark_b200.cage import build_cage_device
    with pytest.raises(Exception):
        build_cage_device(np.zeros((4, 3), np.float32), [[0, 1, 2, 3]])


def test_level_counts_api(lib):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    w = configs.torus_quads()
    m = w.cage.as_cc_mesh()
    arr = (N.LevelCounts * 5)()
    assert lib.ccs_LevelCounts_cuda(ctypes.byref(m), 4, arr) == 0
    assert [arr[d].H for d in range(5)] == [2048 * 4 ** d for d in range(5)]
    assert arr[4].cumH == sum(2048 * 4 ** d for d in range(1, 4))
    assert lib.ccs_MaxSupportedDepth_cuda(ctypes.byref(m)) >= 9
