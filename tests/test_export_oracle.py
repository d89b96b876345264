"""The OBJ-export restatement (oracle.export_obj_text) against the
reference's own ExportToObj (examples/subd_cpu.c:22-115, compiled into
oracle/_ref by oracle/Makefile) on the oracle's refinement: byte for byte, at
every depth, with 16- and 12-byte records, including values whose "%f" text
ends in a rounding tie."""
import os

import numpy as np
import pytest

from oracle import oracle, refimpl


def _cage():
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.cage import build_cage
    w = configs.mixed_torus(nu=8, nv=6, strip=3, depth=2, seed=3)
    pts = np.array(w.points, np.float32)
    # exact ties at the sixth decimal (k / 128), signed zeros, large and tiny values
    pts[:8, 0] = [0.0078125, -0.0078125, 0.0234375, -0.0, 3.0e9, -1.0e-7, 123456.789, 2.5e-6]
    return build_cage(pts, w.faces, w.uvs, w.face_uvs, w.crease_tags)


@pytest.mark.skipif(not refimpl.export_available(), reason="reference not built")
@pytest.mark.parametrize("stride", [4, 3])
def test_export_restatement_matches_reference(tmp_path, stride):
    cage = _cage()
    D = 2
    he, cr, pts = oracle.refine(cage, D, "scatter", np.float32, stride)
    for d in range(D + 1):
        path = str(tmp_path / ("ref_%d.obj" % d))
        refimpl.export_obj(cage, d, D, he, pts, path, uv=stride == 4)
        got = oracle.export_obj_text(cage, d, he, pts, uv=stride == 4)
        assert open(path, "rb").read() == got, d
