"""Edge cases of the cage and the depth: single faces (every edge a boundary),
a triangle, a pentagon, two faces sharing one edge, a creased single quad
with UVs, and subds of depth 1 and 2 (the cage step alone; the cage step and
the two-launch depth-1 step, no one-launch steps).

Against the oracle: topology, creases and UV codes bit-exact; points
bit-exact on the deterministic path and within 1e-5 on the default path, for
the scatter and gather rules; and the adjoint against the FP64 oracle's
transposed operator on one of them.
"""
import numpy as np
import pytest

from conftest import gpu_available, rel_err

pytestmark = pytest.mark.gpu

TOL_POINTS = 1e-5


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def _cages():
    from conftest import small_cages
    return small_cages()


def _gpu(cage, depth, mode, flags=0):
    from halfedgecatmullclark_b200.subd import Subd
    with Subd(cage, depth, flags) as s:
        s.refine(mode)
        s.download()
        return s.halfedges().copy(), s.creases().copy(), s.points().copy()


def _compare(name, cage, depth, mode):
    """Every difference from the oracle, as text (empty when all agree)."""
    from halfedgecatmullclark_b200 import _native as N
    from oracle import oracle
    out = []
    ohe, ocr, opts = oracle.refine(cage, depth, mode, np.float32, 4)
    for label, flags in (("deterministic", N.FLAG_DETERMINISTIC), ("default", 0)):
        he, cr, pts = _gpu(cage, depth, mode, flags)
        bad = np.nonzero(np.any(he[:, :3] != ohe[:, :3], axis=1))[0]
        if bad.size:
            out.append("%s d%d %s %s: %d records differ, first %d: %s vs %s"
                       % (name, depth, mode, label, bad.size, bad[0], he[bad[0]], ohe[bad[0]]))
        if cage.U > 0 and not np.array_equal(he[:, 3], ohe[:, 3]):
            out.append("%s d%d %s %s: UV codes differ" % (name, depth, mode, label))
        if not np.array_equal(cr.view(np.uint8), ocr.view(np.uint8)):
            out.append("%s d%d %s %s: creases differ (%s vs %s)"
                       % (name, depth, mode, label, cr[:4], ocr[:4]))
        if label == "deterministic":
            if not np.array_equal(pts.view(np.uint32), opts.view(np.uint32)):
                i = int(np.argmax(np.any(pts != opts, axis=1)))
                out.append("%s d%d %s %s: points not bit-exact (rel %.3g), first %d: %s vs %s"
                           % (name, depth, mode, label, rel_err(pts, opts), i, pts[i], opts[i]))
        elif rel_err(pts, opts) > TOL_POINTS:
            out.append("%s d%d %s %s: points rel err %.3g" % (name, depth, mode, label, rel_err(pts, opts)))
    return out


@pytest.mark.parametrize("depth", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["scatter", "gather"])
def test_small_cages_match_oracle(depth, mode):
    diffs = []
    for name, cage in _cages():
        diffs += _compare(name, cage, depth, mode)
    assert not diffs, "\n".join(diffs)


def test_small_cage_adjoint_matches_fp64_transpose():
    """<S x, y> = <x, S^T y>: the CUDA adjoint of the creased single quad at
    depth 3 against the FP64 oracle's forward, column by column."""
    import torch
    from halfedgecatmullclark_b200.subd import Subd
    from halfedgecatmullclark_b200.torch_ext import refine_points
    from oracle import oracle
    name, cage = _cages()[-1]
    depth = 3
    with Subd(cage, depth) as s:
        s.refine_scatter()
        s.download()
        he, cr = s.halfedges().copy(), s.creases().copy()
        x = torch.tensor(cage.vertex_points, device="cuda", requires_grad=True)
        p = refine_points(x, s)
        g = torch.randn_like(p, generator=torch.Generator("cuda").manual_seed(3))
        (p * g).sum().backward()
        grad = x.grad.double().cpu().numpy()
    gy = g.double().cpu().numpy()
    dense = np.zeros_like(grad)
    for v in range(cage.V):
        for c in range(3):
            e = np.zeros((cage.V, 3), np.float64)
            e[v, c] = 1.0
            col = oracle.refine_points(cage, depth, he, cr, "scatter", np.float64, cage_points=e)
            dense[v, c] = float((col * gy).sum())
    assert np.abs(grad - dense).max() <= 1e-5 * max(np.abs(dense).max(), 1.0), name
