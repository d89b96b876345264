"""Generate tests/golden/reference_digests.json from the reference itself.

Runs the reference's own ccs_Refine_* (compiled from its sources into
oracle/_ref by `make -C oracle ref`, single-threaded so the float sums are
in halfedge order) on the seeded synthetic cages used by the tests, on the
edge-case cages of tests/conftest.py (depths 1-4) and on the reference's
sample .ccm cages, and records SHA-256 digests of the
refined halfedges, creases and points, plus the per-depth counts.  The
tests compare the oracle against these digests, which pins the oracle on
machines where the reference is not available.

It also copies the sample .ccm cages to tests/golden/_ccm/ (untracked) so
that a copy of the working tree carries them.

Usage:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from halfedgecatmullclark_b200 import ccm, configs  # noqa: E402
from oracle import refimpl  # noqa: E402

REF = os.environ.get("CCS_REFERENCE_DIR", "/root/reference")
MESHES = os.path.join(REF, "examples", "meshes")
MODES = ["scatter", "gather", "nocreases_scatter", "nocreases_gather"]


def golden_workloads():
    """The seeded cages the digests cover (kept small: seconds of CPU)."""
    return [
        configs.torus_quads(depth=4),
        configs.mixed_torus(nu=16, nv=12, strip=6, depth=3, seed=1),
        configs.mixed_torus(nu=10, nv=9, strip=4, depth=4, seed=2),
        configs.height_grid(n=12, depth=3, seed=3),
        configs.fitting_cage(nu=12, nv=10, depth=3, seed=4),
    ]


def digest(arr) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


def topo_digest(he, uv: bool) -> str:
    return digest(he if uv else he[:, :3])


def entry(cage, depth):
    out = {"H0": cage.H, "depth": depth, "modes": {}}
    for mode in MODES:
        he, cr, pts = refimpl.refine(cage, depth, mode)
        out["modes"][mode] = {"halfedges": topo_digest(he, cage.U > 0), "creases": digest(cr),
                              "points": digest(pts)}
    return out


def main():
    if not refimpl.available():
        raise SystemExit("build the reference first: make -C oracle ref")
    refimpl.set_threads(1)
    res = {"generator": "tests/golden/make_golden.py", "workloads": {}, "ccm": {}, "small": {}}
    for w in golden_workloads():
        key = "%s_H%d_d%d" % (w.name, w.cage.H, w.depth)
        res["workloads"][key] = entry(w.cage, w.depth)
    # the edge-case cages (single faces, two faces, a creased quad with UVs)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import small_cages
    for name, cage in small_cages():
        for depth in (1, 2, 3, 4):
            res["small"]["%s_d%d" % (name, depth)] = entry(cage, depth)
    if os.path.isdir(MESHES):
        os.makedirs(os.path.join(HERE, "_ccm"), exist_ok=True)
        for name in sorted(os.listdir(MESHES)):
            if not name.endswith(".ccm"):
                continue
            shutil.copy(os.path.join(MESHES, name), os.path.join(HERE, "_ccm", name))
            cage = ccm.load(os.path.join(MESHES, name))
            e = entry(cage, 2)
            r = refimpl.lib()
            m = refimpl._MeshRef(cage)
            import ctypes
            addr = ctypes.addressof(m.m)
            e["counts"] = {k: [int(getattr(r, fn)(addr, d)) for d in range(6)] for k, fn in (
                ("H", "ccm_HalfedgeCountAtDepth"), ("F", "ccm_FaceCountAtDepth"),
                ("E", "ccm_EdgeCountAtDepth"), ("V", "ccm_VertexCountAtDepth"),
                ("C", "ccm_CreaseCountAtDepth"), ("cumH", "ccs_CumulativeHalfedgeCountAtDepth"),
                ("cumF", "ccs_CumulativeFaceCountAtDepth"), ("cumE", "ccs_CumulativeEdgeCountAtDepth"),
                ("cumV", "ccs_CumulativeVertexCountAtDepth"), ("cumC", "ccs_CumulativeCreaseCountAtDepth"))}
            res["ccm"][name] = e
    with open(os.path.join(HERE, "reference_digests.json"), "w") as fh:
        json.dump(res, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "reference_digests.json"))


if __name__ == "__main__":
    main()
