"""Per-halfedge normals of the finest level (ccs_HalfedgeNormals_cuda)
against the float64 restatement of glsl/CatmullClark_Scatter.glsl:931-960,
evaluated on the same refined points.  Tolerance: 5e-5 absolute per
component (fp32 cross products and an approximate reciprocal square root
against float64)."""
import numpy as np
import pytest

from conftest import ccm_paths, gpu_available

pytestmark = pytest.mark.gpu

TOL = 5e-5


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def _cases(small_workloads):
    from halfedgecatmullclark_b200 import ccm
    out = [(w.name, w.cage, w.depth) for w in small_workloads]
    for p in ccm_paths()[:3]:
        out.append((p.rsplit("/", 1)[-1], ccm.load(p), 2))
    return out


@pytest.mark.parametrize("flags", [0, 1])          # 16-byte records, CCS_FLAG_NO_UV
@pytest.mark.parametrize("smooth", [False, True])
def test_normals_match_oracle(small_workloads, smooth, flags):
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    for name, cage, depth in _cases(small_workloads):
        with Subd(cage, depth, flags) as s:
            s.refine("scatter")
            s.download()
            s.synchronize()
            n = s.normals(smooth).cpu().numpy()
            he = s.halfedges()[s.level_slice(depth, "H")]
            P = s.points()[s.level_slice(depth, "V")]
        ref = oracle.halfedge_normals(he, P, smooth)
        ok = np.isfinite(ref).all(axis=1)                # degenerate faces have no normal
        assert ok.mean() > 0.99, name
        err = np.abs(n[ok] - ref[ok]).max()
        assert err <= TOL, (name, smooth, err)


def test_normals_of_explicit_points():
    """`points` given: the normals follow them, not the subd's own points."""
    import torch
    from halfedgecatmullclark_b200 import configs, torch_ext
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    w = configs.mixed_torus(nu=12, nv=10, strip=4, depth=3, seed=5)
    with Subd(w.cage, w.depth) as s:
        s.refine("scatter")
        s.synchronize()
        s.set_stream(torch.cuda.current_stream())
        cp = torch.tensor(np.asarray(w.cage.vertex_points, np.float32).reshape(-1, 3) * 1.5, device="cuda")
        pts = torch_ext.refine_points(cp, s)
        n = s.normals(True, points=pts).cpu().numpy()
        s.download()
        he = s.halfedges()[s.level_slice(w.depth, "H")]
        P = pts.cpu().numpy()[s.level_slice(w.depth, "V")]
    ref = oracle.halfedge_normals(he, P, True)
    assert np.abs(n - ref).max() <= TOL
