"""Every level of the largest workloads against the reference itself.

Config 2 (the mixed-crease torus with UVs, depth 6: 95 M refined halfedges)
and config 3 (the 256x256 height-field grid, depth 5: 393 M refined
halfedges, 6.3 GB of records) are refined on the GPU and compared, depth by
depth, with the reference's own ccs_Refine_Scatter (CatmullClark.h:3060-3064,
compiled from its sources into oracle/_ref, OpenMP on every host core) on the
same cage:

* halfedge records (twin, edge, vertex and, with UVs, the UV code) and
  creases (next, prev, sharpness bits) byte for byte;
* default points (float atomics in the GPU's order) within 1e-5 of the
  largest coordinate (max-norm relative error, the bar of every parity test);
* the deterministic pass bit for bit against the reference's points pass run
  on one thread (ccs_RefineVertexPoints_Scatter, :2631-2643): its sums in
  halfedge order, the FP32 order the oracle restates.

The comparisons run on the device in chunks: the reference's arrays are
uploaded slice by slice from its own memory (zero-copy views), so the host
holds the reference's hierarchy and nothing more.

The reference's sample cages run at the depths its CPU benchmark uses
(examples/subd_cpu.c:194-204: Bigguy 5, ArmorGuy 4 with 300 non-quads, 7,101
creases and UVs, Imrod 4 with interior valence-2 vertices) in all four point
modes, against the reference's entry point of the same mode.
"""
import os

import numpy as np
import pytest

from conftest import ccm_paths, gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL_POINTS = 1e-5
CHUNK = 1 << 23          # rows per upload (128 MB of 16-byte records)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("oracle/_ref not built (the reference compiled from its sources)")
    from halfedgecatmullclark_b200 import build
    build.build()
    refimpl.set_threads(os.cpu_count() or 1)
    yield
    refimpl.set_threads(os.cpu_count() or 1)


def _first_diff(gpu, ref, cols):
    """Index of the first row where gpu[:, :cols] differs from ref[:, :cols]
    (gpu: CUDA tensor, ref: numpy view with the same rows), or -1."""
    import torch
    n = gpu.shape[0]
    assert ref.shape[0] == n, (ref.shape, gpu.shape)
    for i0 in range(0, n, CHUNK):
        i1 = min(n, i0 + CHUNK)
        r = torch.from_numpy(np.ascontiguousarray(ref[i0:i1])).to(gpu.device)
        ne = (gpu[i0:i1, :cols] != r[:, :cols]).any(dim=1)
        if bool(ne.any()):
            return i0 + int(torch.nonzero(ne)[0, 0])
    return -1


def _point_err(gpu, ref):
    """(max |p - p_ref|, max |p_ref|) over the rows, in float64."""
    import torch
    num, den = 0.0, 0.0
    for i0 in range(0, gpu.shape[0], CHUNK):
        i1 = min(gpu.shape[0], i0 + CHUNK)
        r = torch.from_numpy(np.ascontiguousarray(ref[i0:i1])).to(gpu.device, torch.float64)
        num = max(num, float((gpu[i0:i1].double() - r).abs().max()))
        den = max(den, float(r.abs().max()))
    return num, den


def _compare_levels(s, ref, uv, points="tolerance"):
    """Depth by depth: records and creases bit-exact; points within
    TOL_POINTS ("tolerance"), bit-exact ("exact") or not at all (None).
    Returns the max-norm relative error of the points over all depths."""
    import torch
    arr = s.device_arrays()
    cols = 4 if uv else 3
    num, den = 0.0, 0.0
    for d in range(1, s.depth + 1):
        sl = s.level_slice(d, "H")
        i = _first_diff(arr["halfedges"][sl], ref["halfedges"][sl], cols)
        assert i < 0, "depth %d: halfedge record %d differs" % (d, i)
        sl = s.level_slice(d, "C")
        i = _first_diff(arr["creases"][sl], ref["creases"][sl], 3)
        assert i < 0, "depth %d: crease %d differs" % (d, i)
        sl = s.level_slice(d, "V")
        if points == "exact":
            i = _first_diff(arr["points"][sl].view(torch.int32), ref["points"][sl].view(np.int32), 3)
            assert i < 0, "depth %d: point %d not bit-exact" % (d, i)
        elif points == "tolerance":
            n_, d_ = _point_err(arr["points"][sl], ref["points"][sl])
            num, den = max(num, n_), max(den, d_)
    if points == "tolerance":
        err = num / (den if den > 0 else 1.0)
        assert err <= TOL_POINTS, "default points: max-norm relative error %.3g" % err
        return err
    return 0.0


def _full_size(w, *, uv):
    """The workload's every level against the reference: default pass
    (multi-threaded reference), then the deterministic pass (one-thread
    reference points pass)."""
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import refimpl
    cores = os.cpu_count() or 1
    refimpl.set_threads(cores)
    r = refimpl.RefSubd(w.cage, w.depth)
    try:
        r.refine("scatter")
        ref = r.views()
        with Subd(w.cage, w.depth, N.FLAG_PAGEABLE_HOST) as s:
            assert s.cumH == r.cumH and s.cumC == r.cumC and s.cumV == r.cumV
            s.refine_scatter()
            s.synchronize()
            err = _compare_levels(s, ref, uv, "tolerance")
        # the reference's points pass on one thread: halfedge-order sums
        refimpl.set_threads(1)
        r.call("ccs_RefineVertexPoints_Scatter")
        refimpl.set_threads(cores)
        with Subd(w.cage, w.depth, N.FLAG_PAGEABLE_HOST | N.FLAG_DETERMINISTIC) as s:
            s.refine_scatter()
            s.synchronize()
            _compare_levels(s, ref, uv, "exact")
    finally:
        refimpl.set_threads(cores)
        r.close()
    return err


def test_mixed_torus_depth6_every_level_vs_reference():
    """Config 2 at its full depth 6: 95.1 M refined halfedges with UV codes and
    crease chains, every level against the reference."""
    from halfedgecatmullclark_b200 import configs
    w = configs.mixed_torus()
    assert w.depth == 6 and w.cage.U > 0
    err = _full_size(w, uv=True)
    print("mixed_torus depth 6: default points max-norm rel err vs reference %.3g" % err)


def test_mixed_torus_depth6_default_steps_vs_reference_steps():
    """The default pass's two largest steps (depth 4 -> 5 and 5 -> 6: 17.8 M
    parent halfedges in the last) against the reference's step rules
    (oracle.step_points, pinned to the reference) applied to the pass's own
    previous level: face and edge points bit for bit, vertex points within
    2e-6 -- for the full refine and for the points-only call."""
    from conftest import check_steps
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    w = configs.mixed_torus()
    with Subd(w.cage, w.depth) as s:
        s.refine_scatter()
        s.download()
        he, cr, pts = s.halfedges(), s.creases(), s.points()
        check_steps(w.cage, w.depth, he, cr, pts, True, steps=[4, 5])
        s.refine_vertex_points("scatter")
        s.download()
        check_steps(w.cage, w.depth, he, cr, s.points(), True, steps=[4, 5])


def test_height_grid_depth5_every_level_vs_reference():
    """Config 3 at its full depth 5: 393 M refined halfedges (6.3 GB of
    records), where 64-bit byte offsets meet int32 element ids, every level
    against the reference."""
    from halfedgecatmullclark_b200 import configs
    w = configs.height_grid()
    assert w.depth == 5
    err = _full_size(w, uv=w.cage.U > 0)
    print("height_grid depth 5: default points max-norm rel err vs reference %.3g" % err)


SAMPLE_DEPTHS = {"Bigguy.ccm": 5, "ArmorGuy.ccm": 4, "Imrod.ccm": 4}
POINTS_PASS = {"scatter": "ccs_RefineVertexPoints_Scatter",
               "nocreases_scatter": "ccs_RefineVertexPoints_NoCreases_Scatter"}


def _sample_cages():
    return [(os.path.basename(p), p) for p in ccm_paths() if os.path.basename(p) in SAMPLE_DEPTHS]


@pytest.mark.parametrize("mode", ["scatter", "gather", "nocreases_scatter", "nocreases_gather"])
def test_sample_cages_at_benchmark_depths(mode):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import ccm
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import refimpl
    cages = _sample_cages()
    if len(cages) < len(SAMPLE_DEPTHS):
        pytest.skip("the reference's sample cages are not present")
    cores = os.cpu_count() or 1
    for name, path in cages:
        cage = ccm.load(path)
        depth = SAMPLE_DEPTHS[name]
        refimpl.set_threads(cores)
        r = refimpl.RefSubd(cage, depth)
        try:
            r.refine(mode)
            ref = r.views()
            # the gather rules sum in a fixed order on any thread count: the
            # default GPU pass equals them bit for bit
            with Subd(cage, depth) as s:
                s.refine(mode)
                s.synchronize()
                _compare_levels(s, ref, cage.U > 0, "exact" if mode.endswith("gather") else "tolerance")
            if mode in POINTS_PASS:
                refimpl.set_threads(1)
                r.call(POINTS_PASS[mode])
                refimpl.set_threads(cores)
                with Subd(cage, depth, N.FLAG_DETERMINISTIC) as s:
                    s.refine(mode)
                    s.synchronize()
                    _compare_levels(s, ref, cage.U > 0, "exact")
        finally:
            refimpl.set_threads(cores)
            r.close()
