"""Pins the oracle to the reference.

* always: oracle outputs hash to the digests recorded from the reference
  itself (tests/golden/reference_digests.json, tests/golden/make_golden.py);
* when the reference is built (oracle/_ref): bit-for-bit equality with a
  single-threaded reference run in all four point modes, FP64 agreement,
  and the multi-threaded reference within the atomic-order tolerance.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import ROOT, ccm_paths, rel_err

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_digests.json")
MODES = ["scatter", "gather", "nocreases_scatter", "nocreases_gather"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def golden_workloads():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import golden_workloads as gw
    return gw()


def test_oracle_matches_reference_digests():
    from oracle import oracle
    g = golden()["workloads"]
    seen = 0
    for w in golden_workloads():
        key = "%s_H%d_d%d" % (w.name, w.cage.H, w.depth)
        assert key in g, key
        for mode in MODES:
            he, cr, pts = oracle.refine(w.cage, w.depth, mode)
            ref = g[key]["modes"][mode]
            assert digest(he if w.cage.U > 0 else he[:, :3]) == ref["halfedges"], (key, mode)
            assert digest(cr) == ref["creases"], (key, mode)
            assert digest(pts) == ref["points"], (key, mode)
            seen += 1
    assert seen == 20


def test_oracle_matches_reference_digests_small_cages():
    """The edge-case cages at depths 1-4, all four point modes, against the
    reference's digests (no reference build needed)."""
    from conftest import small_cages
    from oracle import oracle
    g = golden()["small"]
    seen = 0
    for name, cage in small_cages():
        for depth in (1, 2, 3, 4):
            ref_modes = g["%s_d%d" % (name, depth)]["modes"]
            for mode in MODES:
                he, cr, pts = oracle.refine(cage, depth, mode)
                ref = ref_modes[mode]
                assert digest(he if cage.U > 0 else he[:, :3]) == ref["halfedges"], (name, depth, mode)
                assert digest(cr) == ref["creases"], (name, depth, mode)
                assert digest(pts) == ref["points"], (name, depth, mode)
                seen += 1
    assert seen == 96


def test_oracle_matches_reference_digests_ccm():
    from halfedgecatmullclark_b200 import ccm
    from oracle import oracle
    paths = ccm_paths()
    if not paths:
        pytest.skip("sample cages not available")
    g = golden()["ccm"]
    for p in paths:
        name = os.path.basename(p)
        cage = ccm.load(p)
        for mode in MODES:
            he, cr, pts = oracle.refine(cage, 2, mode)
            ref = g[name]["modes"][mode]
            assert digest(he if cage.U > 0 else he[:, :3]) == ref["halfedges"], (name, mode)
            assert digest(cr) == ref["creases"]
            assert digest(pts) == ref["points"], (name, mode)


def _need_ref():
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference not built (make -C oracle ref)")
    return refimpl


@pytest.mark.parametrize("mode", MODES)
def test_oracle_bitexact_vs_reference(small_workloads, mode):
    refimpl = _need_ref()
    from halfedgecatmullclark_b200 import ccm
    from oracle import oracle
    refimpl.set_threads(1)
    cages = [(w.cage, w.depth) for w in small_workloads]
    cages += [(ccm.load(p), 3) for p in ccm_paths()[:4]]
    for cage, depth in cages:
        he, cr, pts = oracle.refine(cage, depth, mode)
        rhe, rcr, rpts = refimpl.refine(cage, depth, mode)
        cols = 4 if cage.U > 0 else 3
        assert np.array_equal(he[:, :cols], rhe[:, :cols])
        assert np.array_equal(cr.view(np.uint8), rcr.view(np.uint8))
        assert np.array_equal(pts.view(np.uint32), rpts.view(np.uint32))


@pytest.mark.parametrize("mode", MODES)
def test_oracle_bitexact_vs_reference_small_cages(mode):
    """The edge-case cages (single faces, two faces, a creased quad with UVs)
    at depths 1-4: the oracle equals the single-threaded reference."""
    refimpl = _need_ref()
    from conftest import small_cages
    from oracle import oracle
    refimpl.set_threads(1)
    for name, cage in small_cages():
        for depth in (1, 2, 3, 4):
            he, cr, pts = oracle.refine(cage, depth, mode)
            rhe, rcr, rpts = refimpl.refine(cage, depth, mode)
            cols = 4 if cage.U > 0 else 3
            assert np.array_equal(he[:, :cols], rhe[:, :cols]), (name, depth)
            assert np.array_equal(cr.view(np.uint8), rcr.view(np.uint8)), (name, depth)
            assert np.array_equal(pts.view(np.uint32), rpts.view(np.uint32)), (name, depth)


def test_fp64_oracle_close_to_reference_fp64(small_workloads):
    refimpl = _need_ref()
    if not refimpl.available64():
        pytest.skip("fp64 reference not built")
    from oracle import oracle
    refimpl.set_threads(1)
    for w in small_workloads:
        he, cr = oracle.refine_topology(w.cage, w.depth)
        p64 = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64)
        _, _, r64 = refimpl.refine(w.cage, w.depth, "scatter", fp64=True)
        # the reference's double build also refines sharpness in double
        assert rel_err(p64, r64) < 1e-6


def test_multithreaded_reference_within_tolerance(small_workloads):
    refimpl = _need_ref()
    from oracle import oracle
    refimpl.set_threads(os.cpu_count() or 4)
    try:
        for w in small_workloads:
            _, _, pts = oracle.refine(w.cage, w.depth, "scatter")
            _, _, rpts = refimpl.refine(w.cage, w.depth, "scatter")
            assert rel_err(pts, rpts) <= 1e-5
    finally:
        refimpl.set_threads(1)


def test_gather_vs_scatter_caveat():
    """The reference's gather and scatter rules differ at interior valence-2
    vertices of quad levels (branch order :2481 vs :2598); the oracle keeps
    both behaviours."""
    _need_ref()
    from halfedgecatmullclark_b200 import ccm
    from oracle import oracle
    paths = [p for p in ccm_paths() if p.endswith("Imrod.ccm")]
    if not paths:
        pytest.skip("Imrod.ccm not available")
    cage = ccm.load(paths[0])
    _, _, s = oracle.refine(cage, 2, "scatter")
    _, _, g = oracle.refine(cage, 2, "gather")
    assert rel_err(s, g) > 1e-4


def test_maps_are_consistent(small_workloads):
    """ccs_EdgeToHalfedgeID / ccs_VertexPointToHalfedgeID restatements."""
    from oracle import oracle
    for w in small_workloads[:3]:
        he, _ = oracle.refine_topology(w.cage, w.depth)
        cnt = oracle.counts(w.cage, w.depth)
        for d in range(1, w.depth + 1):
            lv = he[cnt["cumH"][d - 1]: cnt["cumH"][d - 1] + cnt["H"][d]]
            for e in range(0, cnt["E"][d], max(1, cnt["E"][d] // 200)):
                h = oracle.edge_to_halfedge(w.cage, e, d)
                assert lv[h, 1] == e
            for v in range(0, cnt["V"][d], max(1, cnt["V"][d] // 200)):
                h = oracle.vertex_to_halfedge(w.cage, v, d)
                assert lv[h, 2] == v


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
def test_step_points_compose_to_the_full_pass(small_workloads, mode):
    """oracle.step_points (one step of the scatter rules on given level-d
    points) applied depth by depth reproduces the full points pass bit for
    bit, and the per-step checker passes it and catches a planted error in
    an edge point and in a vertex point."""
    from conftest import check_steps
    from oracle import oracle
    creased = mode == "scatter"
    for w in small_workloads:
        he, cr, pts = oracle.refine(w.cage, w.depth, mode)
        acc = np.zeros_like(pts)
        for d in range(w.depth):
            acc = oracle.step_points(w.cage, w.depth, he, cr, acc, d, creased)
        assert np.array_equal(acc.view(np.uint32), pts.view(np.uint32)), w.name
        check_steps(w.cage, w.depth, he, cr, pts, creased, steps=range(w.depth))
    cnt = oracle.counts(w.cage, w.depth)
    d = w.depth - 1
    edge_row = cnt["cumV"][d] + cnt["V"][d + 1] - 1
    bad = pts.copy()
    bad[edge_row, 0] = np.nextafter(bad[edge_row, 0], np.float32(np.inf))
    with pytest.raises(AssertionError, match="not bit-exact"):
        check_steps(w.cage, w.depth, he, cr, bad, creased, steps=[d])
    bad = pts.copy()
    bad[cnt["cumV"][d], 1] += np.float32(1e-3) * np.abs(pts).max()
    with pytest.raises(AssertionError, match="vertex points"):
        check_steps(w.cage, w.depth, he, cr, bad, creased, steps=[d])
