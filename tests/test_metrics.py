"""The vertex-class counts behind the exact pass's algorithmic bytes
(`metrics.kernel_bytes("exact_points" | "old_vertices")`), checked against
the level counts and the oracle's refined topology: at depth d >= 2 the
vertices that are not older than depth d-1 number F(d-1) + E(d-1) (the
structural count the byte formulas use), the ring walks of the vertices
below V(d-1) visit H(d-1) = H / 4 members and those below V(d-2) H(d-2) =
H / 16, and moving the centres and edge midpoints of depth d-2 faces from
the walks to the per-face kernel moves exactly their points' 24 bytes.
"""
import numpy as np
import pytest

from conftest import small_cages


def _cages():
    from halfedgecatmullclark_b200 import configs
    out = [(name, cage) for name, cage in small_cages()]
    out.append(("mixed_torus", configs.mixed_torus(nu=10, nv=9, strip=4, depth=4, seed=2, with_uv=True).cage))
    out.append(("height_grid", configs.height_grid(n=12, depth=4, seed=3).cage))
    return out


@pytest.mark.parametrize("name,cage", _cages(), ids=[c[0] for c in _cages()])
def test_exact_pass_byte_counts_follow_the_levels(name, cage):
    from halfedgecatmullclark_b200 import metrics
    from halfedgecatmullclark_b200.subd import level_counts
    from oracle import oracle
    depth = 5
    lv = level_counts(cage, depth)
    cnt = oracle.counts(cage, depth)
    he, _ = oracle.refine_topology(cage, depth)
    for d in range(2, depth):
        L = lv[d]
        H = L["H"]
        assert [L[k] for k in ("H", "V", "F", "E", "C")] == [cnt[k][d] for k in ("H", "V", "F", "E", "C")]
        V1, V2 = lv[d - 1]["V"], lv[d - 2]["V"]
        # the structural count of the newer vertices is exact
        assert L["V"] - (H // 16 + (L["E"] - H // 4) // 2) == V1, (name, d)
        for k in ("exact_points", "old_vertices"):
            assert metrics.kernel_bytes(k, L, 16) == metrics.kernel_bytes(k, L, 16, units=V1), (name, d, k)
        # ring members: child-0 halfedges whose vertex is older
        start = cnt["cumH"][d - 1]
        vx = he[start:start + H, 2]
        assert int(np.sum(vx < V1)) == H // 4 == lv[d - 1]["H"], (name, d)
        assert int(np.sum(vx < V2)) == H // 16 == lv[d - 2]["H"], (name, d)
        if d >= 3:
            moved = metrics.kernel_bytes("exact_points", L, 16, units=V2) - \
                metrics.kernel_bytes("exact_points", L, 16, units=V1)
            assert moved == 24 * (V1 - V2), (name, d)
            assert metrics.kernel_bytes("old_vertices", L, 16, units=V2) == \
                2 * 16 * (H // 16) + 24 * (H // 16) + 24 * V2, (name, d)
