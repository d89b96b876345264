"""Source compatibility: a C program written with the reference's own calls
(ccs_Create, ccs_Refine_Scatter, ccs_Release, and a call through a function
pointer as examples/subd_cpu.c's Bench() makes) and include/ccs_cuda_compat.h,
compiled with gcc and linked against lib/libccs_cuda.so, leaves in
subd->halfedges / subd->vertexPoints what the oracle computes."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available, rel_err

pytestmark = pytest.mark.gpu

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "ccs_cuda.h"
#include "ccs_cuda_compat.h"

static void Bench(void (*refine)(cc_Subd *), cc_Subd *subd) { refine(subd); }

int main(int argc, char **argv)
{
    const int depth = atoi(argv[2]);
    const long cumH = atol(argv[3]), cumV = atol(argv[4]);
    cc_Mesh *cage = ccs_LoadCage_cuda(argv[1]);
    if (!cage) return 10;
    cc_Subd *subd = ccs_Create(cage, depth);
    if (!subd) return 11;
    ccs_Refine_Scatter(subd);
    if (ccs_LastError_cuda() != CCS_OK) return 12;
    Bench(&ccs_RefineVertexPoints_Scatter, subd);
    if (ccs_LastError_cuda() != CCS_OK) return 13;
    FILE *f = fopen(argv[5], "wb");
    if (!f) return 14;
    fwrite(subd->halfedges, 16, (size_t)cumH, f);
    fwrite(subd->vertexPoints, 12, (size_t)cumV, f);
    fclose(f);
    ccs_Release(subd);
    ccs_ReleaseCage_cuda(cage);
    return 0;
}
"""


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def test_reference_calls_through_the_compat_header(tmp_path):
    from halfedgecatmullclark_b200 import _native as N, ccm, configs
    from halfedgecatmullclark_b200.subd import level_counts
    from oracle import oracle
    w = configs.mixed_torus(nu=12, nv=10, strip=4, depth=3, seed=7)
    cage_path = str(tmp_path / "cage.ccm")
    ccm.save(w.cage, cage_path)
    src = tmp_path / "prog.c"
    src.write_text(PROGRAM)
    exe = str(tmp_path / "prog")
    libdir = os.path.dirname(N.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c11", "-O1", "-I" + os.path.join(ROOT, "include"), str(src),
                        "-L" + libdir, "-lccs_cuda", "-Wl,-rpath," + libdir, "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = level_counts(w.cage, w.depth)
    cumH = sum(l["H"] for l in L[1:])
    cumV = sum(l["V"] for l in L[1:])
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, cage_path, str(w.depth), str(cumH), str(cumV), out],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    raw = np.fromfile(out, np.uint8)
    he = raw[:16 * cumH].view(np.int32).reshape(-1, 4)
    pts = raw[16 * cumH:].view(np.float32).reshape(-1, 3)
    ohe, ocr, opts = oracle.refine(w.cage, w.depth, "scatter", np.float32, 4)
    assert np.array_equal(he, ohe)
    assert rel_err(pts, opts) <= 1e-5
