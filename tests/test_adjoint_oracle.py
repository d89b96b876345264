"""The oracle's transposed point rule, checked in FP64 three ways:
dot-product test, central finite differences (step 1e-6) and the dense
operator built column by column from forward refinements."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def case():
    from halfedgecatmullclark_b200 import configs
    from oracle import oracle
    w = configs.mixed_torus(nu=7, nv=6, strip=3, depth=3, seed=3)
    he, cr = oracle.refine_topology(w.cage, w.depth)
    return w, he, cr


def forward64(w, he, cr, x):
    from oracle import oracle
    return oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64, cage_points=x)


def test_dot_product(case):
    from oracle import oracle
    w, he, cr = case
    rng = np.random.default_rng(0)
    x = rng.normal(size=(w.cage.V, 3))
    y = rng.normal(size=(forward64(w, he, cr, x).shape[0], 3))
    lhs = float(np.sum(forward64(w, he, cr, x) * y))
    rhs = float(np.sum(x * oracle.adjoint(w.cage, w.depth, he, cr, y)))
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))


def test_finite_differences(case):
    from oracle import oracle
    w, he, cr = case
    rng = np.random.default_rng(1)
    x0 = w.cage.vertex_points.astype(np.float64)
    target = forward64(w, he, cr, x0 + rng.normal(0, 0.05, x0.shape))

    def loss(x):
        return float(np.mean((forward64(w, he, cr, x) - target) ** 2))
    r = forward64(w, he, cr, x0) - target
    g = oracle.adjoint(w.cage, w.depth, he, cr, 2.0 * r / r.size)
    h = 1e-6
    for v in rng.choice(w.cage.V, 16, replace=False):
        for k in range(3):
            xp = x0.copy()
            xm = x0.copy()
            xp[v, k] += h
            xm[v, k] -= h
            fd = (loss(xp) - loss(xm)) / (2 * h)
            assert abs(fd - g[v, k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9


def test_dense_operator(case):
    from oracle import oracle
    w, he, cr = case
    V = w.cage.V
    n = forward64(w, he, cr, np.zeros((V, 3))).shape[0]
    S = np.zeros((n, V))
    for j in range(V):
        e = np.zeros((V, 3))
        e[j, 0] = 1.0
        S[:, j] = forward64(w, he, cr, e)[:, 0]
    rng = np.random.default_rng(2)
    y = rng.normal(size=(n, 3))
    g = oracle.adjoint(w.cage, w.depth, he, cr, y)
    assert np.allclose(g, S.T @ y, rtol=1e-12, atol=1e-12)
    # the rule acts on each coordinate alike (S (x) I3)
    x = rng.normal(size=(V, 3))
    assert np.allclose(forward64(w, he, cr, x), S @ x, rtol=1e-12, atol=1e-12)


def test_dense_operator_small_cages():
    """The edge-case cages (single faces, two faces, a creased quad with UVs)
    at depths 1-4: the oracle's adjoint is the transpose of its forward,
    exactly the dense operator built column by column."""
    from conftest import small_cages
    from oracle import oracle
    rng = np.random.default_rng(2)
    for name, cage in small_cages():
        for depth in (1, 2, 3, 4):
            he, cr = oracle.refine_topology(cage, depth)

            def fwd(x):
                return oracle.refine_points(cage, depth, he, cr, "scatter", np.float64, cage_points=x)
            y = rng.normal(size=(fwd(cage.vertex_points.astype(np.float64)).shape[0], 3))
            g = oracle.adjoint(cage, depth, he, cr, y)
            dense = np.zeros_like(g)
            for v in range(cage.V):
                for c in range(3):
                    e = np.zeros((cage.V, 3))
                    e[v, c] = 1.0
                    dense[v, c] = float(np.sum(fwd(e) * y))
            assert np.abs(g - dense).max() <= 1e-12 * max(1.0, np.abs(dense).max()), (name, depth)
