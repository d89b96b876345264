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


def test_cage_fitting_adam_converges():
    import torch
    from halfedgecatmullclark_b200 import configs
    w = configs.fitting_cage(depth=3)
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
        first = first if first is not None else float(loss)
    assert float(loss) < 0.1 * first
