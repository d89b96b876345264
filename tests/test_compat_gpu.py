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


PROGRAMS = {k: os.path.join(ROOT, "oracle", "_ref", k) for k in ("subd_cpu_ref", "subd_cpu_cuda", "subd_cpu_cuda_det")}


def _run_program(exe, cage_path, depth, workdir, threads=None):
    """examples/subd_cpu.c's command line: <mesh.ccm> <maxDepth> <exportObj>;
    it writes subd_<d>.obj for d = 0..maxDepth into its working directory."""
    os.makedirs(workdir, exist_ok=True)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([exe, cage_path, str(depth), "1"], cwd=workdir, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    assert "All done!" in r.stdout
    return [os.path.join(workdir, "subd_%d.obj" % d) for d in range(depth + 1)]


@pytest.mark.parametrize("cage_name,depth", [("ArmorGuy.ccm", 3), ("Bigguy.ccm", 4)])
def test_reference_program_through_the_compat_header(tmp_path, cage_name, depth):
    """The drop-in with the reference's own program: examples/subd_cpu.c
    (:1-281), compiled unchanged but for include/ccs_cuda_compat.h after
    CatmullClark.h and linked to libccs_cuda.so (oracle/Makefile, target
    subd_cpu), runs its four Bench() passes and its OBJ export (:263-273) on a
    sample cage.  Its subd_<d>.obj files equal those of the same program built
    against the reference alone: byte for byte when both sum the points in
    one order (CCS_FLAG_DETERMINISTIC here, one OpenMP thread there); with the
    default flags (float atomics on both sides) every "vt" and "f" line byte
    for byte and the "v" coordinates within 1e-5 of the largest one (plus the
    1e-6 step of "%f")."""
    from conftest import ccm_paths
    for exe in PROGRAMS.values():
        if not os.path.exists(exe):
            pytest.skip("oracle/_ref programs not built (make -C oracle subd_cpu)")
    paths = [p for p in ccm_paths() if os.path.basename(p) == cage_name]
    if not paths:
        pytest.skip("the reference's sample cages are not present")
    cage = paths[0]
    ref1 = _run_program(PROGRAMS["subd_cpu_ref"], cage, depth, str(tmp_path / "ref1"), threads=1)
    det = _run_program(PROGRAMS["subd_cpu_cuda_det"], cage, depth, str(tmp_path / "det"))
    for a, b in zip(det, ref1):
        with open(a, "rb") as fa, open(b, "rb") as fb:
            assert fa.read() == fb.read(), "%s differs from the reference program's" % os.path.basename(a)
    refn = _run_program(PROGRAMS["subd_cpu_ref"], cage, depth, str(tmp_path / "refn"))
    dflt = _run_program(PROGRAMS["subd_cpu_cuda"], cage, depth, str(tmp_path / "dflt"))
    for a, b in zip(dflt, refn):
        with open(a, "rb") as fa, open(b, "rb") as fb:
            la, lb = fa.read().split(b"\n"), fb.read().split(b"\n")
        assert len(la) == len(lb)
        va = [x for x in la if x.startswith(b"v ")]
        vb = [x for x in lb if x.startswith(b"v ")]
        assert [x for x in la if not x.startswith(b"v ")] == [x for x in lb if not x.startswith(b"v ")]
        pa = np.array([x.split()[1:] for x in va], np.float64)
        pb = np.array([x.split()[1:] for x in vb], np.float64)
        assert pa.shape == pb.shape and pa.shape[0] > 0
        assert np.abs(pa - pb).max() <= 1e-5 * np.abs(pb).max() + 1.5e-6, os.path.basename(a)
