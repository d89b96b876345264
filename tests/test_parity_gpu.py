"""Parity of the CUDA refinement with the oracle (and the reference itself).

Bar: topology, creases and UV codes bit-exact; points bit-exact on every
path whose sums follow the reference's one-thread order (the deterministic
flag, the gather rules), and within 1e-5 of the largest coordinate (max-norm
relative error) for the default scatter path, whose float atomics sum in the
GPU's order.  Errors against the FP64 oracle of the same rule are reported
alongside.
"""
import numpy as np
import pytest

from conftest import ccm_paths, check_steps, gpu_available, rel_err

pytestmark = pytest.mark.gpu

TOL_POINTS = 1e-5


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def gpu_refine(cage, depth, mode="scatter", flags=0):
    from halfedgecatmullclark_b200.subd import Subd
    with Subd(cage, depth, flags) as s:
        s.refine(mode)
        s.download()
        return s.halfedges(), s.creases(), s.points()


def oracle_refine(cage, depth, mode="scatter", stride=4):
    from oracle import oracle
    return oracle.refine(cage, depth, mode, np.float32, stride)


def check_topology(cage, he, cr, ohe, ocr):
    assert np.array_equal(he[:, :3], ohe[:, :3]), "halfedge topology differs"
    if cage.U > 0 and he.shape[1] == 4:
        assert np.array_equal(he[:, 3], ohe[:, 3]), "UV codes differ"
    assert np.array_equal(cr.view(np.uint8), ocr.view(np.uint8)), "creases differ"


def all_cages(small_workloads):
    from halfedgecatmullclark_b200 import ccm
    out = [(w.name + "_d%d" % w.depth, w.cage, w.depth) for w in small_workloads]
    for p in ccm_paths():
        out.append((p.rsplit("/", 1)[-1], ccm.load(p), 2))
    return out


MODES = ["scatter", "gather", "nocreases_scatter", "nocreases_gather"]


@pytest.mark.parametrize("mode", MODES)
def test_refine_matches_oracle(small_workloads, mode):
    from halfedgecatmullclark_b200 import _native as N
    for name, cage, depth in all_cages(small_workloads):
        ohe, ocr, opts = oracle_refine(cage, depth, mode)
        # deterministic scatter / gather: same summation order as the oracle
        he, cr, pts = gpu_refine(cage, depth, mode, N.FLAG_DETERMINISTIC)
        check_topology(cage, he, cr, ohe, ocr)
        assert np.array_equal(pts.view(np.uint32), opts.view(np.uint32)), \
            "%s %s: deterministic points not bit-exact (rel err %.3g)" % (name, mode, rel_err(pts, opts))
        # default path (float atomics for the scatter rules)
        he, cr, pts = gpu_refine(cage, depth, mode)
        check_topology(cage, he, cr, ohe, ocr)
        err = rel_err(pts, opts)
        assert err <= TOL_POINTS, "%s %s: rel err %.3g" % (name, mode, err)
        if mode.endswith("gather"):
            assert np.array_equal(pts.view(np.uint32), opts.view(np.uint32))


def test_error_against_fp64_oracle(small_workloads):
    """FP32 error of GPU and reference-order FP32 against the FP64 rule."""
    from oracle import oracle
    for name, cage, depth in all_cages(small_workloads):
        he, cr, pts = gpu_refine(cage, depth, "scatter")
        p64 = oracle.refine_points(cage, depth, he, cr, "scatter", np.float64)
        o32 = oracle.refine_points(cage, depth, he, cr, "scatter", np.float32)
        e_gpu = rel_err(pts, p64)
        e_ref = rel_err(o32, p64)
        rms = float(np.sqrt(np.mean((pts.astype(np.float64) - p64) ** 2)) / np.abs(p64).max())
        assert e_gpu <= TOL_POINTS, "%s: %.3g" % (name, e_gpu)
        # the GPU is as accurate as the reference's own FP32 order
        assert e_gpu <= 4 * e_ref + 1e-7, "%s: gpu %.3g vs fp32 order %.3g" % (name, e_gpu, e_ref)
        assert rms <= e_gpu + 1e-12


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
def test_default_steps_match_reference_steps(small_workloads, mode):
    """Each step of the default pass (the one-launch steps at depth >= 2 with
    their float atomics, both the full refine and the points-only call)
    reproduces the reference's step arithmetic on its own previous level
    (the cage step, a sparse map with double sums, within tolerance)."""
    from halfedgecatmullclark_b200.subd import Subd
    for w in small_workloads:
        with Subd(w.cage, w.depth) as s:
            s.refine(mode)
            s.download()
            he, cr, pts = s.halfedges(), s.creases(), s.points()
            check_steps(w.cage, w.depth, he, cr, pts, mode == "scatter", steps=range(w.depth))
            s.refine_vertex_points(mode)
            s.download()
            check_steps(w.cage, w.depth, he, cr, s.points(), mode == "scatter", steps=range(w.depth))


def test_separate_entry_points(small_workloads):
    """ccs_RefineHalfedges/Creases/VertexUvs/VertexPoints_* one by one."""
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    for w in small_workloads:
        ohe, ocr = oracle.refine_topology(w.cage, w.depth)
        with Subd(w.cage, w.depth) as s:
            s.refine_halfedges()
            s.refine_creases()
            s.refine_vertex_uvs()
            for mode in MODES:
                s.refine_vertex_points(mode)
                s.download()
                he, cr, pts = s.halfedges(), s.creases(), s.points()
                check_topology(w.cage, he, cr, ohe, ocr)
                opts = oracle.refine_points(w.cage, w.depth, ohe, ocr, mode, np.float32)
                assert rel_err(pts, opts) <= TOL_POINTS, (w.name, mode)


def test_no_uv_layout(small_workloads):
    """12-byte records: the CC_DISABLE_UV build of cc_Halfedge_SemiRegular."""
    from halfedgecatmullclark_b200 import _native as N
    for w in small_workloads:
        ohe, ocr, opts = oracle_refine(w.cage, w.depth, "scatter", stride=3)
        he, cr, pts = gpu_refine(w.cage, w.depth, "scatter", N.FLAG_NO_UV | N.FLAG_DETERMINISTIC)
        assert he.shape[1] == 3
        assert np.array_equal(he, ohe)
        assert np.array_equal(cr.view(np.uint8), ocr.view(np.uint8))
        assert np.array_equal(pts.view(np.uint32), opts.view(np.uint32))


def test_points_before_topology_is_an_error(small_workloads):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.subd import Subd
    w = small_workloads[0]
    with Subd(w.cage, w.depth) as s:
        with pytest.raises(N.CcsError) as ei:
            s.refine_vertex_points("scatter")
        assert ei.value.code == -6


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
def test_fused_and_separate_passes_agree(small_workloads, mode):
    """Fused level kernels == the reference's pass structure, bit for bit."""
    from halfedgecatmullclark_b200 import _native as N
    for w in small_workloads:
        a = gpu_refine(w.cage, w.depth, mode, N.FLAG_DETERMINISTIC)
        b = gpu_refine(w.cage, w.depth, mode, N.FLAG_DETERMINISTIC | N.FLAG_SEPARATE_PASSES)
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (w.name, mode)
        c = gpu_refine(w.cage, w.depth, mode, N.FLAG_SEPARATE_PASSES)
        assert rel_err(c[2], a[2]) <= TOL_POINTS
        # the default fused path: same topology, points within tolerance
        f = gpu_refine(w.cage, w.depth, mode)
        for x, y in zip(a[:2], f[:2]):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (w.name, mode)
        assert rel_err(f[2], a[2]) <= TOL_POINTS


def test_graph_and_direct_launch_agree(small_workloads):
    from halfedgecatmullclark_b200 import _native as N
    w = small_workloads[1]
    a = gpu_refine(w.cage, w.depth, "scatter", N.FLAG_DETERMINISTIC)
    b = gpu_refine(w.cage, w.depth, "scatter", N.FLAG_DETERMINISTIC | N.FLAG_NO_GRAPH)
    for x, y in zip(a, b):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_repeated_refine_is_stable(small_workloads):
    """A second refine on the same subd (graph replay) gives the same result."""
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.subd import Subd
    w = small_workloads[2]
    with Subd(w.cage, w.depth, N.FLAG_DETERMINISTIC) as s:
        s.refine_scatter()
        s.download()
        p1 = s.points()
        s.refine_scatter()
        s.download()
        assert np.array_equal(p1.view(np.uint32), s.points().view(np.uint32))


def test_upload_cage_points(small_workloads):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    w = small_workloads[1]
    rng = np.random.default_rng(7)
    newp = (w.cage.vertex_points + rng.normal(0, 0.05, w.cage.vertex_points.shape)).astype(np.float32)
    with Subd(w.cage, w.depth, N.FLAG_DETERMINISTIC) as s:
        s.refine_scatter()
        s.upload_cage_points(newp)
        s.refine_vertex_points("scatter")
        s.download()
        he, cr = s.halfedges(), s.creases()
        opts = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float32, cage_points=newp)
        assert np.array_equal(s.points().view(np.uint32), opts.view(np.uint32))


def test_against_reference_build():
    """The reference's own multi-threaded ccs_Refine_Scatter, when built."""
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("oracle/_ref not built")
    from halfedgecatmullclark_b200 import configs
    w = configs.mixed_torus(nu=24, nv=20, strip=8, depth=4, seed=5)
    refimpl.set_threads(refimpl.max_threads())
    rhe, rcr, rpts = refimpl.refine(w.cage, w.depth, "scatter")
    he, cr, pts = gpu_refine(w.cage, w.depth, "scatter")
    check_topology(w.cage, he, cr, rhe, rcr)
    assert rel_err(pts, rpts) <= TOL_POINTS


@pytest.mark.slow
def test_mixed_torus_depth6_properties():
    """Full-size mixed-crease workload: size-independent checks + a sampled
    slice against the oracle's rule."""
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    w = configs.mixed_torus()
    with Subd(w.cage, w.depth) as s:
        s.refine_scatter()
        s.download()
        he, cr, pts = s.halfedges(), s.creases(), s.points()
    cnt = oracle.counts(w.cage, w.depth)
    assert he.shape[0] == cnt["cumH"][w.depth]
    # every level: twins are an involution, vertex ids in range
    for d in range(1, w.depth + 1):
        sl = slice(cnt["cumH"][d - 1], cnt["cumH"][d - 1] + cnt["H"][d])
        lv = he[sl]
        tw = lv[:, 0]
        ok = tw >= 0
        assert np.all(lv[tw[ok], 0] == np.nonzero(ok)[0])
        assert lv[:, 2].min() >= 0 and lv[:, 2].max() < cnt["V"][d]
    # the first four levels, recomputed by the oracle over the GPU topology
    ohe, ocr = oracle.refine_topology(w.cage, 4)
    assert np.array_equal(he[:ohe.shape[0]], ohe)
    o32 = oracle.refine_points(w.cage, 4, ohe, ocr, "scatter", np.float32)
    assert rel_err(pts[:o32.shape[0]], o32) <= TOL_POINTS
    assert np.isfinite(pts).all()
    # the deterministic pass at full size: the first four levels bit for bit
    from halfedgecatmullclark_b200 import _native as N
    with Subd(w.cage, w.depth, N.FLAG_DETERMINISTIC) as s:
        s.refine_scatter()
        s.download()
        dpts = s.points()
    assert np.array_equal(dpts[:o32.shape[0]].view(np.uint32), o32.view(np.uint32))
    assert rel_err(dpts, pts) <= TOL_POINTS


@pytest.mark.slow
def test_height_grid_depth5_properties():
    """Config 3 at full size (256x256 height-field grid with diagonal splits
    and creases, depth 5: 393 M refined halfedges, 6.3 GB of records), checked
    on the device arrays: twins an involution and vertex ids in range at
    every level, finite points; the first three levels equal to the oracle
    (topology and creases bit-exact, default points within 1e-5, the
    deterministic pass bit for bit)."""
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    from oracle import oracle
    w = configs.height_grid()
    assert w.depth == 5
    ohe, ocr = oracle.refine_topology(w.cage, 3)
    o32 = oracle.refine_points(w.cage, 3, ohe, ocr, "scatter", np.float32)
    cnt = oracle.counts(w.cage, w.depth)
    for flags in (N.FLAG_PAGEABLE_HOST, N.FLAG_PAGEABLE_HOST | N.FLAG_DETERMINISTIC):
        with Subd(w.cage, w.depth, flags) as s:
            s.refine_scatter()
            s.synchronize()
            arr = s.device_arrays()
            he, cr, pts = arr["halfedges"], arr["creases"], arr["points"]
            assert he.shape[0] == cnt["cumH"][w.depth]
            for d in range(1, w.depth + 1):
                lv = he[s.level_slice(d, "H")]
                tw = lv[:, 0].long()
                ok = tw >= 0
                assert torch.equal(lv[tw[ok], 0].long(), torch.nonzero(ok).squeeze(1))
                assert int(lv[:, 2].min()) >= 0 and int(lv[:, 2].max()) < cnt["V"][d]
                del tw, ok
            assert bool(torch.isfinite(pts).all())
            n = ohe.shape[0]
            assert np.array_equal(he[:n, :3].cpu().numpy(), ohe[:, :3])
            assert np.array_equal(cr[:ocr.shape[0]].cpu().numpy().view(np.uint8).reshape(-1),
                                  ocr.view(np.uint8).reshape(-1))
            p = pts[:o32.shape[0]].cpu().numpy()
            if flags & N.FLAG_DETERMINISTIC:
                assert np.array_equal(p.view(np.uint32), o32.view(np.uint32))
            else:
                assert rel_err(p, o32) <= TOL_POINTS


def test_profiled_refine_times_the_graph_and_matches():
    """With profiling on, a refine replays a graph of its own with event
    record nodes: every launch and every step d -> d+1 comes back with a
    positive device time, the steps' records cover depths 0..D-1, and the
    results equal those of the unprofiled graph (deterministic pass: bit for
    bit); a second profiled refine gives the same records again."""
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import Subd
    w = configs.mixed_torus(nu=12, nv=10, strip=4, depth=4, seed=7)
    with Subd(w.cage, w.depth, N.FLAG_DETERMINISTIC) as s:
        st = torch.cuda.Stream()
        s.set_stream(st)
        s.refine_scatter()
        s.download()
        he0, pts0 = s.halfedges(), s.points()
        s.set_profiling(True)
        counts = []
        for _ in range(2):
            s.refine_scatter()
            recs = s.read_profile(1 << 12)
            counts.append(len(recs))
            assert recs and all(r["ms"] > 0 for r in recs)
            steps = sorted(r["level"] for r in recs if r["kernel"] == "step")
            assert steps == list(range(w.depth))
        s.set_profiling(False)
        assert counts[0] == counts[1]
        s.download()
        assert np.array_equal(s.halfedges(), he0)
        assert np.array_equal(s.points().view(np.uint32), pts0.view(np.uint32))
