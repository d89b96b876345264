"""OBJ export formatted on the GPU (ccs_ExportObj_cuda) against the
reference's ExportToObj (examples/subd_cpu.c:22-115) on the same refined
arrays: byte for byte, every depth, 16- and 12-byte records, default and
deterministic points.  Where the reference is not built, against the
restatement oracle.export_obj_text (itself pinned to the reference in
tests/test_export_oracle.py)."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def _expected(cage, d, D, he, pts, uv, tmp_path):
    from oracle import oracle, refimpl
    if refimpl.export_available():
        path = str(tmp_path / "ref.obj")
        refimpl.export_obj(cage, d, D, he, pts, path, uv=uv)
        return open(path, "rb").read()
    return oracle.export_obj_text(cage, d, he, pts, uv=uv)


@pytest.mark.parametrize("flags", [0, 1, 4])        # default, CCS_FLAG_NO_UV, CCS_FLAG_DETERMINISTIC
def test_export_matches_reference_bytes(tmp_path, flags):
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    w = configs.mixed_torus(nu=10, nv=8, strip=4, depth=3, seed=7)
    D = 3
    with Subd(w.cage, D, flags) as s:
        s.refine("scatter")
        s.download()
        he, pts = s.halfedges(), s.points()
        for d in range(D + 1):
            path = str(tmp_path / ("gpu_%d.obj" % d))
            s.export_obj(path, d)
            got = open(path, "rb").read()
            assert got == _expected(w.cage, d, D, he, pts, s.record_words == 4, tmp_path), (flags, d)


def test_export_refuses_bad_depth(tmp_path):
    from halfedgecatmullclark_b200 import _native as N, configs
    from halfedgecatmullclark_b200.subd import Subd
    w = configs.torus_quads(depth=2)
    with Subd(w.cage, 2) as s:
        s.refine("scatter")
        for d in (-1, 3):
            assert N.lib().ccs_ExportObj_cuda(s.ptr, d, str(tmp_path / "x.obj").encode()) == -1
