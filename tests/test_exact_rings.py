"""The index identities the exact vertex pass's per-face kernel relies on
(`tile_face_exact` in csrc/ccs_tiles.cuh), checked on the oracle's refined
levels of closed, open and non-quad cages.

At depth d >= 3 the kernel sums, besides the parent quads' centres and
edge midpoints, the older vertices that are the centre and the edge
midpoints of a grandparent face G (a depth d-2 face; its 16 depth-d faces
are 16 G .. 16 G + 15).  It never walks their rings: it takes the members,
the twin side's faces and edges, and the ownership of each midpoint from
the numbering of the refined records.  These tests check, for every such
vertex, that the members the kernel derives are exactly the halfedges
whose vertex it is, that the derived edge ids are the records' own, that
each vertex is claimed by exactly one thread, and that the ring walks left
to `old_vertex_item` (ids below V(d-2)) take exactly the other corners.
The topology rules these follow are CatmullClark.h:2749-2796.
"""
import numpy as np
import pytest

from conftest import small_cages


def _qnext(h):
    return (h & ~3) | ((h + 1) & 3)


def _qprev(h):
    return (h & ~3) | ((h - 1) & 3)


def _cages():
    from halfedgecatmullclark_b200 import configs
    out = [(name, cage, 5) for name, cage in small_cages()]
    out.append(("mixed_torus", configs.mixed_torus(nu=10, nv=9, strip=4, depth=4, seed=2, with_uv=True).cage, 4))
    out.append(("height_grid", configs.height_grid(n=12, depth=4, seed=3).cage, 4))
    return out


def _level(he, cnt, d):
    start = cnt["cumH"][d - 1]
    rec = he[start:start + cnt["H"][d]]
    return rec[:, 0].astype(np.int64), rec[:, 1].astype(np.int64), rec[:, 2].astype(np.int64)


@pytest.mark.parametrize("name,cage,depth", _cages(), ids=[c[0] for c in _cages()])
def test_grandparent_corner_rings_follow_the_numbering(name, cage, depth):
    from oracle import oracle
    cnt = oracle.counts(cage, depth)
    he, _ = oracle.refine_topology(cage, depth)
    for d in range(3, depth + 1):
        tw, ed, vx = _level(he, cnt, d)
        nF = cnt["H"][d] // 4
        V2, V1 = cnt["V"][d - 2], cnt["V"][d - 1]
        f = np.arange(nF, dtype=np.int64)
        j = f & 3
        g = f >> 2
        C = vx[4 * f]
        tw3 = tw[4 * f + 3]
        # the ring of every vertex: its halfedges, sorted (older vertices'
        # members are child-0 halfedges)
        order = np.argsort(vx, kind="stable")
        vs = vx[order]
        first = np.searchsorted(vs, np.arange(cnt["V"][d]), "left")
        last = np.searchsorted(vs, np.arange(cnt["V"][d]), "right")

        def ring(v):
            return np.sort(order[first[v]:last[v]])

        # corners 0: vertices of depth d-2 (the ring walks), corners 1-3: the rest
        assert np.all(C[j == 0] < V2), (name, d)
        assert np.all((C[j != 0] >= V2) & (C[j != 0] < V1)), (name, d)
        # G's centre: corner 2 of its four quads, members child 0 of faces 16 G + 4 J + 2
        cen = f[j == 2]
        G = cen >> 4
        assert np.array_equal(C[cen].reshape(-1, 4), np.repeat(C[cen][::4, None], 4, axis=1)), (name, d)
        for k in range(0, cen.size, 4):
            want = 4 * (16 * G[k] + 4 * np.arange(4) + 2)
            assert np.array_equal(ring(C[cen[k]]), want), (name, d, k)
        # G's edge midpoints: corner 1 of quad J, corner 3 of quad J+1
        f1 = f[j == 1]
        g1 = g[j == 1]
        t3 = tw3[j == 1]
        gT = _qprev(t3 >> 4)
        own = (t3 < 0) | (g1 > gT)
        f2 = 4 * _qnext(g1) + 3
        assert np.array_equal(C[f2], C[f1]), (name, d)
        e0 = ed[4 * f1]
        eT1 = 2 * ((e0 >> 1) - g1 + gT) + np.where((gT & 3) == 3, 0, 1)
        claims = np.zeros(cnt["V"][d], np.int64)
        np.add.at(claims, C[f1[own]], 1)
        np.add.at(claims, C[cen[::4]], 1)
        assert np.all(claims[V2:V1] == 1), (name, d)
        assert np.all(claims[:V2] == 0), (name, d)
        for i in np.nonzero(own)[0]:
            members = [4 * f1[i], 4 * f2[i]]
            if t3[i] >= 0:
                m1 = 4 * (4 * gT[i] + 1)
                members += [m1, t3[i]]
                assert ed[m1] == eT1[i], (name, d, i)       # the twin side's inner member
                assert ed[t3[i]] == ed[4 * f1[i] + 3], (name, d, i)
                assert C[m1 >> 2] == C[f1[i]] and vx[t3[i]] == C[f1[i]], (name, d, i)
            else:
                # boundary: (j, 3)'s edge has no member; f2's prev edge is f1's own
                assert tw[4 * f1[i]] >= 0 and tw[4 * f2[i]] < 0, (name, d, i)
                assert ed[4 * f2[i] + 3] == ed[4 * f1[i]], (name, d, i)
            assert np.array_equal(ring(C[f1[i]]), np.sort(members)), (name, d, i)
