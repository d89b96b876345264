"""The per-halfedge normal restatement (oracle.halfedge_normals) on meshes
whose normals are known in closed form: a planar grid (every normal is the
plane's, boundary halfedges included) and a torus (smooth normals point away
from the tube's centre line)."""
import numpy as np

from halfedgecatmullclark_b200 import configs
from halfedgecatmullclark_b200.cage import build_cage
from oracle import oracle


def grid_cage(nx, ny):
    """Open planar nx x ny quad grid in z = 0."""
    x, y = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    pts = np.stack([x, y, np.zeros_like(x)], -1).reshape(-1, 3).astype(np.float32)
    vid = lambda i, j: i * (ny + 1) + j
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)]
             for i in range(nx) for j in range(ny)]
    return build_cage(pts, faces)


def torus_cage(nu, nv):
    """Noise-free quad torus, major radius 1, minor radius 0.3."""
    pts = configs._torus_points(nu, nv, 1.0, 0.3).astype(np.float32)
    vid = lambda i, j: (i % nu) * nv + (j % nv)
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)]
             for i in range(nu) for j in range(nv)]
    return build_cage(pts, faces)


def _finest(cage, depth):
    he, cr, pts = oracle.refine(cage, depth, "scatter", real=np.float64)
    hs = oracle.level_slice(cage, depth, depth, "H")
    vs = oracle.level_slice(cage, depth, depth, "V")
    return he[hs], pts[vs]


def test_planar_grid_normals_are_vertical():
    cage = grid_cage(6, 4)
    he, P = _finest(cage, 2)
    for smooth in (False, True):
        n = oracle.halfedge_normals(he, P, smooth)
        assert np.allclose(np.abs(n[:, 2]), 1.0, atol=1e-12)
        assert np.allclose(n[:, 2], n[0, 2])                 # one consistent orientation


def test_torus_smooth_normals_point_out_of_the_tube():
    cage = torus_cage(12, 8)
    he, P = _finest(cage, 2)
    n = oracle.halfedge_normals(he, P, True)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-12)
    v = P[he[:, 2]]
    rho = np.hypot(v[:, 0], v[:, 1])
    R = 0.5 * (rho.max() + rho.min())                       # tube centre radius
    centre = np.stack([v[:, 0] * R / rho, v[:, 1] * R / rho, np.zeros_like(rho)], axis=1)
    radial = v - centre
    radial /= np.linalg.norm(radial, axis=1, keepdims=True)
    cos = np.sum(n * radial, axis=1)
    assert abs(np.mean(np.sign(cos))) == 1.0                # all one side
    assert np.min(np.abs(cos)) > 0.9
