"""The CUDA adjoint and the torch.autograd function.

References: the FP64 oracle adjoint (itself checked against the FP64 dense
operator and finite differences in test_adjoint_oracle.py), FP64 central
finite differences (step 1e-6) of the cage-fitting loss on 64 random cage
vertices, and the dot-product identity <S x, y> = <x, S^T y>.
"""
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


def surface(w):
    from halfedgecatmullclark_b200.torch_ext import SubdivisionSurface
    return SubdivisionSurface(w.cage, w.depth)


def test_adjoint_matches_fp64_oracle(small_workloads):
    import torch
    from halfedgecatmullclark_b200.torch_ext import RefinePoints
    from oracle import oracle
    for w in small_workloads:
        s = surface(w)
        x = torch.tensor(w.cage.vertex_points, device="cuda", requires_grad=True)
        pts = RefinePoints.apply(x, s.subd)
        g = torch.randn_like(pts)
        pts.backward(g)
        he, cr = oracle.refine_topology(w.cage, w.depth)
        ref = oracle.adjoint(w.cage, w.depth, he, cr, g.double().cpu().numpy())
        assert rel_err(x.grad.cpu().numpy(), ref) <= 1e-5, w.name
        # forward through the device entry point == the C ABI refine
        p64 = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64)
        assert rel_err(pts.detach().cpu().numpy(), p64) <= 1e-5


def test_dot_product_identity(small_workloads):
    import torch
    from halfedgecatmullclark_b200.torch_ext import refine_points
    w = small_workloads[1]
    s = surface(w)
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((w.cage.V, 3), device="cuda", generator=gen, requires_grad=True)
    y = torch.randn((s.subd.cumV, 3), device="cuda", generator=gen)
    p = refine_points(x, s.subd)
    (p * y).sum().backward()
    lhs = float((p.detach().double() * y.double()).sum())
    rhs = float((x.detach().double() * x.grad.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * max(1.0, abs(lhs))


def test_finite_differences_fitting_loss():
    """FP64 central differences of mean ||P_D - T||^2 at 64 cage vertices."""
    import torch
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.torch_ext import level
    from oracle import oracle
    w = configs.fitting_cage(depth=3)
    s = surface(w)
    rng = np.random.default_rng(0)
    x0 = w.cage.vertex_points.astype(np.float64)
    he, cr = oracle.refine_topology(w.cage, w.depth)
    sl = s.subd.level_slice(w.depth, "V")

    def fwd64(x):
        return oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64, cage_points=x)[sl]
    target = fwd64(x0 + rng.normal(0, 0.05, x0.shape))
    x = torch.tensor(x0, dtype=torch.float32, device="cuda", requires_grad=True)
    t = torch.tensor(target, dtype=torch.float32, device="cuda")
    loss = ((s(x) - t) ** 2).mean()
    loss.backward()
    g = x.grad.cpu().numpy()
    n = target.size
    # the loss is quadratic: central differences are exact up to rounding
    verts = rng.choice(w.cage.V, 64, replace=False)
    h = 1e-6
    fd_all, g_all = [], []
    for v in verts:
        for k in range(3):
            xp = x0.copy()
            xm = x0.copy()
            xp[v, k] += h
            xm[v, k] -= h
            fd_all.append((np.mean((fwd64(xp) - target) ** 2) - np.mean((fwd64(xm) - target) ** 2)) / (2 * h))
            g_all.append(g[v, k])
    fd_all, g_all = np.array(fd_all), np.array(g_all)
    assert n > 0
    assert np.abs(fd_all - g_all).max() <= 2e-5 * np.abs(fd_all).max()


def test_dense_operator_gradient():
    """Gradient against the FP64 dense operator, streamed column by column."""
    import torch
    from halfedgecatmullclark_b200 import configs
    from oracle import oracle
    w = configs.mixed_torus(nu=8, nv=7, strip=3, depth=3, seed=6)
    s = surface(w)
    he, cr = oracle.refine_topology(w.cage, w.depth)
    sl = s.subd.level_slice(w.depth, "V")
    rng = np.random.default_rng(3)
    r = rng.normal(size=(sl.stop - sl.start, 3))
    x = torch.tensor(w.cage.vertex_points, device="cuda", requires_grad=True)
    out = s(x)
    out.backward(torch.tensor(r, dtype=torch.float32, device="cuda"))
    dense = np.zeros((w.cage.V, 3))
    for j in range(w.cage.V):
        e = np.zeros((w.cage.V, 3))
        e[j, 0] = 1.0
        col = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64, cage_points=e)[sl, 0]
        dense[j] = col @ r
    assert rel_err(x.grad.cpu().numpy(), dense) <= 1e-5


@pytest.mark.slow
def test_fitting_cage_depth5_gradient_fd_and_dense():
    """Config 4 as stated (2000-face mixed cage, depth 5; loss = mean squared
    distance of the finest points to the refinement of the cage perturbed by
    N(0, 0.05^2)): the CUDA gradient through torch.autograd against FP64
    central differences (step 1e-6) and the FP64 dense operator, streamed one
    basis column at a time, at 64 random cage vertices (the FP64 forwards run
    in a spawn pool of the oracle)."""
    import torch
    from halfedgecatmullclark_b200 import configs
    from oracle import fd
    w = configs.fitting_cage(depth=5)
    assert w.depth == 5 and 1900 <= w.cage.F <= 2100
    target = fd.target(5, seed=0, sigma=0.05)
    verts = np.random.default_rng(7).choice(w.cage.V, 64, replace=False)
    s = surface(w)
    x = torch.tensor(w.cage.vertex_points, device="cuda", requires_grad=True)
    t = torch.tensor(target, dtype=torch.float32, device="cuda")
    loss = ((s(x) - t) ** 2).mean()
    loss.backward()
    g = x.grad.cpu().numpy()[verts]
    fdv, dense = fd.check_gradient(verts, 5, seed=0, sigma=0.05, h=1e-6)
    scale = np.abs(dense).max()
    assert scale > 0
    assert np.abs(fdv - dense).max() <= 1e-6 * scale     # the two FP64 references agree
    assert np.abs(g - dense).max() <= 1e-5 * scale, np.abs(g - dense).max() / scale
    assert np.abs(g - fdv).max() <= 2e-5 * np.abs(fdv).max()


@pytest.mark.parametrize("depth", [3, pytest.param(5, marks=pytest.mark.slow)])
def test_cage_fitting_adam_converges(depth):
    """100 Adam steps of the fitting loss fall by 10x (config 4 is depth 5)."""
    import torch
    from halfedgecatmullclark_b200 import configs
    w = configs.fitting_cage(depth=depth)
    s = surface(w)
    rng = np.random.default_rng(1)
    x0 = torch.tensor(w.cage.vertex_points, device="cuda")
    with torch.no_grad():
        target = s(x0 + torch.tensor(rng.normal(0, 0.05, w.cage.vertex_points.shape), dtype=torch.float32,
                                     device="cuda"))
    x = x0.clone().requires_grad_(True)
    opt = torch.optim.Adam([x], lr=5e-3)
    first = None
    for _ in range(100):
        opt.zero_grad()
        loss = ((s(x) - target) ** 2).mean()
        loss.backward()
        opt.step()
        first = first if first is not None else float(loss.detach())
    assert float(loss.detach()) < 0.1 * first


def _boundary_crease_cage():
    """Open 8x6 quad grid whose boundary is smooth except for one semi-sharp
    segment on the left side, ending at the vertex where a semi-sharp
    interior chain (a full row of edges) starts: an older boundary vertex in
    the crease branch with a creased interior edge.  (Cages built with the
    OBJ converter's conventions sharpen every boundary edge, which puts such
    a vertex in the corner branch; a caller's own cage need not.)"""
    from halfedgecatmullclark_b200.cage import build_cage
    nx, ny = 8, 6
    rng = np.random.default_rng(11)
    x, y = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    pts = np.stack([x, y, 0.3 * rng.normal(size=x.shape)], -1).reshape(-1, 3).astype(np.float32)
    vid = lambda i, j: i * (ny + 1) + j
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)] for i in range(nx) for j in range(ny)]
    tags = [(vid(i, 3), vid(i + 1, 3), 5.0) for i in range(nx)]
    cage = build_cage(pts, faces, crease_tags=tags)
    he = cage.halfedges
    sharp = cage.creases["sharpness"]
    for e, h in enumerate(cage.e2h):
        if he["twinID"][h] < 0:
            a, b = he["vertexID"][h], he["vertexID"][he["nextID"][h]]
            left = a // (ny + 1) == 0 and b // (ny + 1) == 0 and max(a % (ny + 1), b % (ny + 1)) <= 3
            sharp[e] = 4.0 if left else 0.0
    return cage


def _boundary_crease_hits(cage, depth):
    """Child-0 halfedges with a twin whose (older, boundary) vertex has two
    creased edges, valence above 2 and whose own edge is creased: the case
    where the one-pass adjoint reads the twin quad's next edge."""
    from oracle import oracle
    he, cr = oracle.refine_topology(cage, depth)
    hits = 0
    for d in range(2, depth):
        hs = oracle.level_slice(cage, depth, d, "H")
        rec = he[hs]
        C = oracle.counts(cage, depth)["C"][d]
        cs = oracle.level_slice(cage, depth, d, "C")
        sharp = np.zeros(rec.shape[0] * 2 + 16, np.float32)
        sharp[:C] = cr[cs]["sharpness"]
        vold = oracle.counts(cage, depth)["V"][d - 1]
        tw, ed, vx = rec[:, 0], rec[:, 1], rec[:, 2]
        inc = {}
        bnd = np.zeros(int(vx.max()) + 1, bool)
        for h in range(rec.shape[0]):
            inc.setdefault(int(vx[h]), set()).add(int(ed[h]))
            if tw[h] < 0:
                bnd[vx[h]] = True
                nxt = (h & ~3) | ((h + 1) & 3)
                inc.setdefault(int(vx[nxt]), set()).add(int(ed[h]))
                bnd[vx[nxt]] = True
        for h in range(0, rec.shape[0], 4):
            v = int(vx[h])
            if tw[h] < 0 or v >= vold or not bnd[v] or sharp[ed[h]] == 0:
                continue
            n_crease = sum(1 for e in inc[v] if e < C and sharp[e] > 0)
            if n_crease == 2 and len(inc[v]) != 2:
                hits += 1
    return hits


def test_one_pass_adjoint_boundary_crease_branch():
    import torch
    from halfedgecatmullclark_b200.torch_ext import RefinePoints, SubdivisionSurface
    from oracle import oracle
    cage = _boundary_crease_cage()
    depth = 4
    assert _boundary_crease_hits(cage, depth) > 0     # the branch is reached
    s = SubdivisionSurface(cage, depth)
    x = torch.tensor(cage.vertex_points, device="cuda", requires_grad=True)
    pts = RefinePoints.apply(x, s.subd)
    g = torch.randn_like(pts)
    pts.backward(g)
    he, cr = oracle.refine_topology(cage, depth)
    ref = oracle.adjoint(cage, depth, he, cr, g.double().cpu().numpy())
    assert rel_err(x.grad.cpu().numpy(), ref) <= 1e-5


@pytest.mark.slow
def test_fitting_cage_depth5_adjoint():
    """Config 4 at its full depth (2000-face mixed cage, depth 5): the CUDA
    adjoint of a random gradient against the FP64 oracle adjoint."""
    import torch
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.torch_ext import RefinePoints
    from oracle import oracle
    w = configs.fitting_cage(depth=5)
    s = surface(w)
    x = torch.tensor(w.cage.vertex_points, device="cuda", requires_grad=True)
    pts = RefinePoints.apply(x, s.subd)
    g = torch.randn(pts.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    pts.backward(g)
    he, cr = oracle.refine_topology(w.cage, w.depth)
    ref = oracle.adjoint(w.cage, w.depth, he, cr, g.double().cpu().numpy())
    assert rel_err(x.grad.cpu().numpy(), ref) <= 1e-5
