"""Shared test setup.

Markers: ``gpu`` tests need a CUDA device and the built library; everything
else runs on the CPU.  The checker (``oracle/``) is built on demand from its
committed sources with gcc.
"""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference checkout the checker reads, when it is present (never on a
# machine that only runs the GPU tests).  One variable, CCS_REFERENCE_DIR,
# names it for every test and recipe; the default is where the container
# that builds this repository mounts it.
REF = os.environ.get("CCS_REFERENCE_DIR", "/root/reference")
REFERENCE_MESHES = os.path.join(REF, "examples", "meshes")
LOCAL_MESHES = os.path.join(ROOT, "tests", "golden", "_ccm")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and lib/libccs_cuda.so")
    config.addinivalue_line("markers", "slow: larger workloads")


def ccm_paths():
    """Cage fixtures: the reference's sample .ccm files when present.

    They are read from the reference checkout, or from the untracked copy
    under tests/golden/_ccm that tests/golden/make_golden.py makes so that
    they travel with the working tree to a GPU machine.
    """
    for d in (REFERENCE_MESHES, LOCAL_MESHES):
        paths = sorted(glob.glob(os.path.join(d, "*.ccm")))
        if paths:
            return paths
    return []


@pytest.fixture(scope="session")
def small_workloads():
    from halfedgecatmullclark_b200 import configs
    return [
        configs.torus_quads(depth=3),
        configs.mixed_torus(nu=16, nv=12, strip=6, depth=3, seed=1),
        configs.mixed_torus(nu=10, nv=9, strip=4, depth=4, seed=2, with_uv=True),
        configs.height_grid(n=12, depth=3, seed=3),
        configs.fitting_cage(nu=12, nv=10, depth=3, seed=4),
    ]


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def fusable(cage):
    """The twin relation the fused level kernels need: vertex(twin h) ==
    vertex(next h) for every halfedge with a twin (the C ABI's own check)."""
    he = cage.halfedges
    tw = he["twinID"]
    ok = tw >= 0
    return bool(np.all(he["vertexID"][tw[ok]] == he["vertexID"][he["nextID"][ok]]))


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def small_cages():
    """Edge-case cages: single faces (every edge a boundary), a quad and a
    triangle sharing an edge, two quads, and a creased single quad with UVs."""
    from halfedgecatmullclark_b200.cage import build_cage
    rng = np.random.default_rng(11)
    quad = np.array([[0, 0, 0], [1, 0, 0.1], [1, 1, 0], [0, 1, 0.2]], np.float32)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0.3, 0.9, 0.4]], np.float32)
    pent = np.array([[np.cos(a), np.sin(a), 0.1 * i] for i, a in
                     enumerate(np.linspace(0, 2 * np.pi, 5, endpoint=False))], np.float32)
    two = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0.3], [0, 1, 0], [2, 0, 0.1], [2, 1, 0]], np.float32)
    uvs = rng.uniform(0, 1, (4, 2)).astype(np.float32)
    return [
        ("quad", build_cage(quad, [[0, 1, 2, 3]])),
        ("triangle", build_cage(tri, [[0, 1, 2]])),
        ("pentagon", build_cage(pent, [[0, 1, 2, 3, 4]])),
        ("quad_and_triangle", build_cage(two[:5], [[0, 1, 2, 3], [1, 4, 2]])),
        ("two_quads", build_cage(two, [[0, 1, 2, 3], [1, 4, 5, 2]])),
        ("creased_quad_uv", build_cage(quad, [[0, 1, 2, 3]], uvs=uvs, face_uvs=[[0, 1, 2, 3]],
                                       crease_tags=[(0, 1, 1.5)])),
    ]


def check_steps(cage, depth, he, cr, pts, creased, steps=None, tol=2e-6):
    """Steps d -> d+1 (default: all but the cage step, d >= 1) of a default
    (float-atomic) pass against the reference's own step on the pass's
    level-d points: face and edge points bit for bit (their sums have a fixed
    order), vertex points within `tol` of the level's largest coordinate (the
    atomics' order).  The default cage step applies the step as a sparse map
    with double sums, so its face and edge points are only within `tol`."""
    from oracle import oracle
    cnt = oracle.counts(cage, depth)
    for d in (range(1, depth) if steps is None else steps):
        ref = oracle.step_points(cage, depth, he, cr, pts, d, creased)
        a, V0, V1 = cnt["cumV"][d], cnt["V"][d], cnt["V"][d + 1]
        got, want = pts[a:a + V1], ref[a:a + V1]
        if d == 0:
            V0 = V1
        i = np.flatnonzero((got[V0:].view(np.uint32) != want[V0:].view(np.uint32)).any(axis=1))
        assert i.size == 0, "step %d: face/edge point %d not bit-exact" % (d, V0 + i[0])
        scale = float(np.abs(want).max())
        err = float(np.abs(got[:V0].astype(np.float64) - want[:V0]).max()) / scale
        assert err <= tol, "step %d: vertex points off by %.3g" % (d, err)
