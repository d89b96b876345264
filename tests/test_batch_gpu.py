"""Batched refinement: every cage of a batch against the single-mesh path and
the oracle (topology bit-exact; points within 1e-5 by default, bit-exact with
the deterministic flag), the batched adjoint against the single-mesh adjoint,
the autograd function, the bounded grid-barrier wait, and the autotuner's
cache."""
import numpy as np
import pytest

from conftest import gpu_available, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


@pytest.fixture(scope="module")
def workloads():
    from halfedgecatmullclark_b200 import configs
    ws = configs.batch_cages(count=20, fmin=20, fmax=400, dmin=1, dmax=4, seed=3)
    ws.append(configs.mixed_torus(nu=10, nv=8, strip=3, depth=3, seed=4))        # with UVs
    ws.append(configs.torus_quads(nu=8, nv=6, depth=4))
    return ws


@pytest.mark.parametrize("deterministic", [False, True])
def test_batch_refine_matches_oracle(workloads, deterministic):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.batch import Batch
    from oracle import oracle
    flags = N.FLAG_DETERMINISTIC if deterministic else 0
    with Batch([w.cage for w in workloads], [w.depth for w in workloads], flags) as b:
        b.refine()
        b.synchronize()
        for i, w in enumerate(workloads):
            he, cr, pts = b.download(i)
            ohe, ocr, opts = oracle.refine(w.cage, w.depth, "scatter")
            cols = 4 if w.cage.U > 0 else 3
            assert np.array_equal(he[:, :cols], ohe[:, :cols]), w.name
            assert np.array_equal(cr.view(np.uint8), ocr.view(np.uint8)), w.name
            if deterministic:
                assert np.array_equal(pts.view(np.uint32), opts.view(np.uint32)), (w.name, rel_err(pts, opts))
            else:
                assert rel_err(pts, opts) <= 1e-5, (w.name, rel_err(pts, opts))
        # points only, from the kept topology and ring statistics
        b.refine_points()
        b.synchronize()
        for i, w in enumerate(workloads):
            opts = oracle.refine(w.cage, w.depth, "scatter")[2]
            assert rel_err(b.download(i)[2], opts) <= 1e-5, w.name


def test_batch_points_and_adjoint_match_single_mesh(workloads):
    import torch
    from halfedgecatmullclark_b200.batch import Batch
    from halfedgecatmullclark_b200.torch_ext import SubdivisionSurface, refine_points
    rng = np.random.default_rng(5)
    with Batch([w.cage for w in workloads], [w.depth for w in workloads]) as b:
        b.refine()
        arr = b.arrays()
        newp = [(w.cage.vertex_points + rng.normal(0, 0.02, w.cage.vertex_points.shape)).astype(np.float32)
                for w in workloads]
        for i in range(len(workloads)):
            arr["cage_points"][b.cage_slice(i)] = torch.tensor(newp[i], device="cuda")
        b.set_stream(torch.cuda.current_stream())
        b.refine_points()
        grads = torch.randn_like(arr["points"])
        arr["grad_points"].copy_(grads)
        b.adjoint()
        b.synchronize()
        for i, w in enumerate(workloads):
            s = SubdivisionSurface(w.cage, w.depth)
            x = torch.tensor(newp[i], device="cuda", requires_grad=True)
            p = refine_points(x, s.subd)
            # the single-mesh default sums with float atomics: within tolerance
            bp = arr["points"][b.point_slice(i)].cpu().numpy()
            assert rel_err(bp, p.detach().cpu().numpy()) <= 1e-5
            p.backward(grads[b.point_slice(i)])
            assert rel_err(arr["grad_cage_points"][b.cage_slice(i)].cpu().numpy(), x.grad.cpu().numpy()) <= 1e-5


def test_batch_autograd(workloads):
    import torch
    from halfedgecatmullclark_b200 import batch as B
    with B.Batch([w.cage for w in workloads], [w.depth for w in workloads]) as b:
        b.refine()
        x0 = torch.cat([torch.tensor(w.cage.vertex_points) for w in workloads]).cuda()
        x = x0.clone().requires_grad_(True)
        pts = B.refine_points(x, b)
        loss = (pts ** 2).sum()
        loss.backward()
        # the same through two independent forwards (linearity): d/dx sum p^2 = 2 S^T S x
        x2 = x0.clone().requires_grad_(True)
        pts2 = B.refine_points(x2, b)
        (2.0 * pts2.detach() * pts2).sum().backward()
        assert rel_err(x.grad.cpu().numpy(), x2.grad.cpu().numpy()) <= 1e-5


def test_bounded_barrier_wait_reports_timeout(workloads):
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.batch import Batch
    L = N.lib()
    assert L.ccs_BarrierTimeoutSelfTest_cuda() == -5      # gave up and reported
    # the context is still usable
    with Batch([w.cage for w in workloads[:3]], [w.depth for w in workloads[:3]]) as b:
        b.refine()
        b.synchronize()


def test_autotune_writes_and_reuses_cache(workloads, tmp_path, monkeypatch):
    from halfedgecatmullclark_b200 import batch as B
    monkeypatch.setenv("CCS_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    with B.Batch([w.cage for w in workloads], [w.depth for w in workloads]) as b:
        b.refine()
        first = B.autotune(b, candidates=(0, 1, 2), iters=2)
        assert not first["cached"] and (tmp_path / "tune.json").exists()
        again = B.autotune(b, candidates=(0, 1, 2), iters=2)
        assert again["cached"] and again["blocks_per_sm"] == first["blocks_per_sm"]


def test_split_schedule_matches_fused(workloads):
    """One launch per section gives what one cooperative launch per depth gives:
    bit for bit with the deterministic flag (topology, points, adjoint)."""
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200.batch import Batch
    outs = []
    for split in (False, True):
        with Batch([w.cage for w in workloads], [w.depth for w in workloads], N.FLAG_DETERMINISTIC) as b:
            b.set_schedule(0, split)
            b.refine()
            arr = b.arrays()
            gen = torch.Generator(device="cuda").manual_seed(1)
            arr["grad_points"].copy_(torch.randn(arr["grad_points"].shape, device="cuda", generator=gen))
            b.adjoint()
            b.synchronize()
            outs.append((arr["halfedges"].cpu().numpy(), arr["points"].cpu().numpy(),
                         arr["grad_cage_points"].cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))
    assert rel_err(outs[1][2], outs[0][2]) <= 1e-5


@pytest.mark.slow
def test_batch_config5_distribution_matches_reference():
    """64 cages drawn from the batched workload's own distribution (faces
    log-uniform in [50, 5000], mixed triangles / quads / pentagons, 0-10 %
    crease edges with sharpness U[0, 4], depths uniform in {2..6}; about 0.5 G
    refined halfedges), each against the reference's own ccs_Refine_Scatter
    (CatmullClark.h:3060-3064, compiled from its sources): topology and
    creases bit-exact, default points within 1e-5; the deterministic batch bit
    for bit against the reference's points pass on one thread."""
    import os
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.batch import Batch
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("oracle/_ref not built")
    ws = configs.batch_cages(count=64, seed=21)
    assert {w.depth for w in ws} == {2, 3, 4, 5, 6}
    cores = os.cpu_count() or 1
    with Batch([w.cage for w in ws], [w.depth for w in ws]) as b, \
            Batch([w.cage for w in ws], [w.depth for w in ws], N.FLAG_DETERMINISTIC) as bd:
        b.refine()
        bd.refine()
        b.synchronize()
        bd.synchronize()
        for i, w in enumerate(ws):
            refimpl.set_threads(cores)
            r = refimpl.RefSubd(w.cage, w.depth)
            try:
                r.refine("scatter")
                rhe, rcr, rpts = r.halfedges(), r.creases(), r.points()
                he, cr, pts = b.download(i)
                assert np.array_equal(he[:, :3], rhe[:, :3]), w.name
                assert np.array_equal(cr.view(np.uint8), rcr.view(np.uint8)), w.name
                assert rel_err(pts, rpts) <= 1e-5, (w.name, rel_err(pts, rpts))
                refimpl.set_threads(1)
                r.call("ccs_RefineVertexPoints_Scatter")
                dpts = bd.download(i)[2]
                assert np.array_equal(dpts.view(np.uint32), r.points().view(np.uint32)), w.name
            finally:
                refimpl.set_threads(cores)
                r.close()


@pytest.mark.parametrize("split", [True, False])
def test_batch_distance_adjoint_matches_plain(workloads, split):
    """ccs_BatchAdjointDistance_cuda (the finest level of every cage of depth
    >= 3 read as P - T inside its first adjoint step, the other levels set to
    P - T first) equals the plain batched adjoint fed P - T, within the float
    atomics' reordering: cages of depths 1-4, both launch schedules, two calls
    with different targets (the second re-captures the operation's graph)."""
    import torch
    from halfedgecatmullclark_b200.batch import Batch
    with Batch([w.cage for w in workloads], [w.depth for w in workloads]) as b:
        b.set_stream(torch.cuda.current_stream())
        b.refine()
        b.set_schedule(0 if split else 4, split)
        arr = b.arrays()
        gen = torch.Generator(device="cuda").manual_seed(7)
        for _ in range(2):
            T = torch.randn(arr["points"].shape, device="cuda", generator=gen)
            b.refine_points()
            b.adjoint_distance(T)
            b.synchronize()
            got = arr["grad_cage_points"].clone()
            arr["grad_points"].copy_(arr["points"] - T)
            b.adjoint()
            b.synchronize()
            ref = arr["grad_cage_points"].clone()
            assert torch.isfinite(got).all()
            assert rel_err(got.cpu().numpy(), ref.cpu().numpy()) <= 1e-5
