"""Device-side cage build (ccs_BuildCage_cuda) against the host builder
`cage.build_cage`, which is itself compared byte for byte with the
reference's LoadObj (tests/test_cage_io.py): every array of the cage must be
byte-identical, on every workload generator and on edge cases of the
converter's rules (crease tags overriding one another and the boundary
rule, tags with equal ends, isolated vertices, n-gons)."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

FIELDS = ["vertex_points", "uvs", "halfedges", "creases", "v2h", "e2h", "f2h"]


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def same(a, b):
    bad = [f for f in FIELDS if not np.array_equal(np.asarray(getattr(a, f)).view(np.uint8),
                                                   np.asarray(getattr(b, f)).view(np.uint8))]
    return bad


def device(w):
    from halfedgecatmullclark_b200.cage import build_cage_device
    return build_cage_device(w.points, w.faces, w.uvs, w.face_uvs, w.crease_tags)


def test_workload_cages_match_host_builder():
    from halfedgecatmullclark_b200 import configs
    ws = [configs.torus_quads(), configs.mixed_torus(), configs.mixed_torus(nu=7, nv=5, strip=3, seed=9),
          configs.height_grid(n=40, seed=2), configs.fitting_cage()]
    ws += configs.batch_cages(count=24, fmax=3000, seed=5)
    for w in ws:
        assert same(device(w), w.cage) == [], w.name


def test_converter_rules_edge_cases():
    from halfedgecatmullclark_b200.cage import build_cage, build_cage_device
    # a 3x2 grid of quads with a triangle folded over its last column, an
    # isolated vertex (index 12) and tags that override one another, have
    # equal ends, hit a boundary edge and name vertices that share no edge
    pts = np.random.default_rng(3).normal(size=(13, 3)).astype(np.float32)
    vid = lambda i, j: i * 3 + j
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)] for i in range(3) for j in range(2)]
    faces.append([vid(3, 2), vid(3, 1), vid(3, 0)])
    tags = [(vid(1, 0), vid(1, 1), 2.0), (vid(1, 1), vid(1, 0), 3.5), (vid(0, 0), vid(1, 0), 1.0),
            (vid(2, 1), vid(2, 1), 4.0), (vid(0, 0), vid(3, 2), 5.0), (vid(1, 1), vid(2, 1), 0.75)]
    for kw in ({}, {"crease_tags": tags}):
        ref = build_cage(pts, faces, **kw)
        got = build_cage_device(pts, faces, **kw)
        assert same(got, ref) == []
    # n-gons with UVs
    faces = [[0, 1, 2, 3, 4], [0, 4, 5], [4, 3, 6, 5]]
    fuv = [[0, 1, 2, 3, 4], [0, 4, 5], [4, 3, 6, 5]]
    uvs = np.random.default_rng(4).random((7, 2)).astype(np.float32)
    p7 = np.random.default_rng(5).normal(size=(7, 3)).astype(np.float32)
    assert same(build_cage_device(p7, faces, uvs, fuv), build_cage(p7, faces, uvs, fuv)) == []


def test_refused_inputs():
    from halfedgecatmullclark_b200.cage import build_cage_device
    pts = np.zeros((5, 3), np.float32)
    for faces in ([[0, 1]],                         # fewer than 3 corners
                  [[0, 1, 7]],                      # vertex out of range
                  [[0, 1, 2], [0, 1, 3]],           # directed edge 0 -> 1 twice
                  [[0, 1, 1, 2]]):                  # two consecutive corners on one vertex
        with pytest.raises(ValueError):
            build_cage_device(pts, faces)
    with pytest.raises(ValueError):                 # texture index out of range
        build_cage_device(pts, [[0, 1, 2]], np.zeros((2, 2), np.float32), [[0, 1, 2]])


def test_device_built_cage_refines_like_host_built():
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    w = configs.mixed_torus(nu=16, nv=12, strip=6, depth=3, seed=1)
    res = []
    for cage in (w.cage, device(w)):
        with Subd(cage, 3, 4) as s:                 # deterministic: bit-comparable
            s.refine("scatter")
            s.download()
            res.append((s.halfedges(), s.creases(), s.points()))
    for a, b in zip(*res):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
