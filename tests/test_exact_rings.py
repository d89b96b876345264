"""The index identities and the arithmetic of the exact vertex pass's
per-face kernel (`tile_face_exact` in csrc/ccs_tiles.cuh) for the corners it
sums without a ring walk, checked on the oracle's refined levels of closed,
open and non-quad cages.

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
The topology rules these follow are CatmullClark.h:2749-2796.  A float32
restatement of the kernel's statistics, shares and summation order for
those corners then reproduces the reference-order points bit for bit
(the vertex rule of CatmullClark.h:2496-2615, with and without creases).
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


# ---------------------------------------------------------------------------
# The kernel's arithmetic for those corners, restated in float32 numpy (every
# operation an IEEE round-to-nearest float32 operation, no fused multiply-add,
# as the kernels are built), against the reference-order points of the oracle.
# ---------------------------------------------------------------------------
f32 = np.float32


def _fsign(x):
    return np.where(x < 0, f32(-1), np.where(x > 0, f32(1), f32(0))).astype(f32)


def _rule(p, F, E, Ep, vpre, cpre, avgS, bnd, cw, pcw, creased):
    """quad_vertex_rule (CatmullClark.h:2496-2615): one halfedge's share."""
    col = lambda x: np.asarray(x, f32)[:, None]
    if not creased:
        w = f32(1) / vpre
        ws = w * np.where(bnd, f32(0), f32(1)).astype(f32)
        return (col(w) * (p + col(ws) * ((f32(4) * E - F) - f32(3) * p))).astype(f32)
    valence = np.where(bnd, vpre + f32(1), vpre).astype(f32)
    count = np.where(bnd, cpre + cw, cpre).astype(f32)
    corner = p * col(f32(1) / vpre)
    smooth = (F * f32(-1) + E * f32(4)) + p * col(vpre - f32(3))
    smooth = smooth * col(f32(1) / (vpre * vpre))
    q = f32(0.25) * cw
    crease = p * col(q) + E * col(q)
    qp = f32(0.25) * pcw
    crease = np.where(col(bnd), crease + (p * col(qp) + Ep * col(qp)), crease)
    h = avgS * f32(0.5)
    u = np.where(f32(0) > np.where(h < f32(1), h, f32(1)), f32(0), np.where(h < f32(1), h, f32(1))).astype(f32)
    lerp = corner + col(u) * (crease - corner)
    out = np.where(col((count >= 3) | (valence == 2)), corner, np.where(col(count <= 1), smooth, lerp))
    return out.astype(f32)


def _sum_sorted(ids, shares):
    """Shares (k, n, 3) summed from zero in increasing id order (ids (k, n))."""
    order = np.argsort(ids, axis=0, kind="stable")
    acc = np.zeros(shares.shape[1:], f32)
    for r in range(ids.shape[0]):
        acc = (acc + np.take_along_axis(shares, order[r][None, :, None], 0)[0]).astype(f32)
    return acc


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
@pytest.mark.parametrize("name,cage,depth", _cages(), ids=[c[0] for c in _cages()])
def test_grandparent_corner_sums_match_the_reference_order(name, cage, depth, mode):
    from oracle import oracle
    creased = mode == "scatter"
    cnt = oracle.counts(cage, depth)
    he, cr, pts = oracle.refine(cage, depth, mode)
    for d in range(3, depth):
        tw, ed, vx = _level(he, cnt, d)
        s0 = cnt["cumC"][d - 1]
        sharp_d = cr["sharpness"][s0:s0 + cnt["C"][d]]

        def sharp(e):
            """Sharpness of level-d edges: 0 past the crease records, or without creases."""
            e = np.asarray(e, np.int64)
            if not creased:
                return np.zeros(e.shape, f32)
            ok = e < sharp_d.size
            return np.where(ok, sharp_d[np.where(ok, e, 0)], f32(0)).astype(f32)

        P = pts[oracle.level_slice(cage, depth, d, "V")]
        Q = pts[oracle.level_slice(cage, depth, d + 1, "V")]
        Vd, Fd = cnt["V"][d], cnt["F"][d]
        Fp, Ep = Q[Vd:Vd + Fd], Q[Vd + Fd:]
        nF = cnt["H"][d] // 4
        f = np.arange(nF, dtype=np.int64)
        j, g = f & 3, f >> 2
        C = vx[4 * f]
        # G's centres: the lanes j = 2 of quads 0..3, in quad order
        cen = f[j == 2].reshape(-1, 4)
        n = cen.shape[0]
        sc = sharp(ed[4 * cen])                                   # (n, 4)
        tot = np.zeros(n, f32)
        cntz = np.zeros(n, f32)
        for J in range(4):
            tot = (tot + sc[:, J]).astype(f32)
            cntz = (cntz + _fsign(sc[:, J])).astype(f32)
        four = np.full(n, f32(4))
        shares = np.stack([_rule(P[C[cen[:, J]]], Fp[cen[:, J]], Ep[ed[4 * cen[:, J]]], np.zeros((n, 3), f32),
                                 four, cntz, tot, np.zeros(n, bool), _fsign(sc[:, J]), np.zeros(n, f32),
                                 creased) for J in range(4)])
        got = _sum_sorted(np.stack([4 * cen[:, J] for J in range(4)]), shares)
        want = Q[C[cen[:, 0]]]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, mode, d, "centres")
        # G's edge midpoints, summed by the owner of G's halfedge J (lane j = 1)
        f1 = f[j == 1]
        g1 = g[j == 1]
        t3 = tw[4 * f1 + 3]
        gT = _qprev(t3 >> 4)
        own = (t3 < 0) | (g1 > gT)
        f1, g1, t3, gT = f1[own], g1[own], t3[own], gT[own]
        f2 = 4 * _qnext(g1) + 3
        pC = P[C[f1]]
        sa, sb, s3 = sharp(ed[4 * f1]), sharp(ed[4 * f2]), sharp(ed[4 * f1 + 3])
        inner = t3 >= 0
        # interior: four members, the ring's statistics shared by all
        i = inner
        m1 = 4 * (4 * gT[i] + 1)
        eT1 = 2 * ((ed[4 * f1[i]] >> 1) - g1[i] + gT[i]) + np.where((gT[i] & 3) == 3, 0, 1)
        sT = sharp(eT1)
        tot = (((sa[i] + sb[i]).astype(f32) + sT).astype(f32) + s3[i]).astype(f32)
        cn = (((_fsign(sa[i]) + _fsign(sb[i])).astype(f32) + _fsign(sT)).astype(f32) + _fsign(s3[i])).astype(f32)
        k = int(i.sum())
        z3, four, no = np.zeros((k, 3), f32), np.full(k, f32(4)), np.zeros(k, bool)
        zk = np.zeros(k, f32)
        sh = np.stack([
            _rule(pC[i], Fp[f1[i]], Ep[ed[4 * f1[i]]], z3, four, cn, tot, no, _fsign(sa[i]), zk, creased),
            _rule(pC[i], Fp[f2[i]], Ep[ed[4 * f2[i]]], z3, four, cn, tot, no, _fsign(sb[i]), zk, creased),
            _rule(pC[i], Fp[4 * gT[i] + 1], Ep[eT1], z3, four, cn, tot, no, _fsign(sT), zk, creased),
            _rule(pC[i], Fp[t3[i] >> 2], Ep[ed[4 * f1[i] + 3]], z3, four, cn, tot, no, _fsign(s3[i]), zk,
                  creased)])
        got = _sum_sorted(np.stack([4 * f1[i], 4 * f2[i], m1, t3[i]]), sh)
        want = Q[C[f1[i]]]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, mode, d, "inner midpoints")
        # boundary: two members; the ring's edge without a member is (j, 3)'s
        b = ~inner
        k = int(b.sum())
        if k:
            two, yes = np.full(k, f32(2)), np.ones(k, bool)
            aA = (s3[b] + sb[b]).astype(f32)
            cA = (_fsign(s3[b]) + _fsign(sb[b])).astype(f32)
            aB = (s3[b] + sa[b]).astype(f32)
            cB = (_fsign(s3[b]) + _fsign(sa[b])).astype(f32)
            sh = np.stack([
                _rule(pC[b], Fp[f1[b]], Ep[ed[4 * f1[b]]], Ep[ed[4 * f1[b] + 3]], two, cA, aA, yes,
                      _fsign(sa[b]), _fsign(s3[b]), creased),
                _rule(pC[b], Fp[f2[b]], Ep[ed[4 * f2[b]]], Ep[ed[4 * f1[b]]], two, cB, aB, yes,
                      _fsign(sb[b]), _fsign(sa[b]), creased)])
            got = _sum_sorted(np.stack([4 * f1[b], 4 * f2[b]]), sh)
            want = Q[C[f1[b]]]
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, mode, d, "boundary midpoints")


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
@pytest.mark.parametrize("name,cage,depth", _cages(), ids=[c[0] for c in _cages()])
def test_parent_centre_and_midpoint_sums_match_the_reference_order(name, cage, depth, mode):
    """The rest of the kernel's sums, from depth 2: the parent quad's centre
    from the quad's four (j, 2) shares, and the parent edge's midpoint at the
    pair's owner from (j, 1), (j+1, 3) and the twin side's two shares rebuilt
    from its face and edge points."""
    from oracle import oracle
    creased = mode == "scatter"
    cnt = oracle.counts(cage, depth)
    he, cr, pts = oracle.refine(cage, depth, mode)
    for d in range(2, depth):
        tw, ed, vx = _level(he, cnt, d)
        s0 = cnt["cumC"][d - 1]
        sharp_d = cr["sharpness"][s0:s0 + cnt["C"][d]]

        def sharp(e):
            e = np.asarray(e, np.int64)
            if not creased:
                return np.zeros(e.shape, f32)
            ok = e < sharp_d.size
            return np.where(ok, sharp_d[np.where(ok, e, 0)], f32(0)).astype(f32)

        P = pts[oracle.level_slice(cage, depth, d, "V")]
        Q = pts[oracle.level_slice(cage, depth, d + 1, "V")]
        Vd, Fd = cnt["V"][d], cnt["F"][d]
        Fp, Ep = Q[Vd:Vd + Fd], Q[Vd + Fd:]
        nF = cnt["H"][d] // 4
        f = np.arange(nF, dtype=np.int64)
        nxt = f - (f & 3) + ((f + 1) & 3)                          # the next face of the quad
        zn, no, four = np.zeros(nF, f32), np.zeros(nF, bool), np.full(nF, f32(4))
        e0, e1, e2, e3 = ed[4 * f], ed[4 * f + 1], ed[4 * f + 2], ed[4 * f + 3]
        # the shares of (j, 2) at the centre and (j, 3) at M_{j-1}, every face
        sh2 = _rule(P[vx[4 * f + 2]], Fp[f], Ep[e2], Ep[e1], four, zn, zn, no, _fsign(sharp(e2)),
                    _fsign(sharp(e1)), creased)
        bnd3 = tw[4 * f + 3] < 0
        s3, s3x = sharp(e3), sharp(e3 ^ 1)
        avg3 = np.where(bnd3, s3x, (s3 + s3x).astype(f32)).astype(f32)
        cp3 = np.where(bnd3, _fsign(s3x), (_fsign(s3) + _fsign(s3x)).astype(f32)).astype(f32)
        sh3 = _rule(P[vx[4 * f + 3]], Fp[f], Ep[e3], Ep[e2], np.where(bnd3, f32(2), f32(4)).astype(f32), cp3,
                    avg3, bnd3, _fsign(s3), _fsign(sharp(e2)), creased)
        # centres: the quad's four (j, 2) in face order
        q = f[(f & 3) == 0]
        got = _sum_sorted(np.stack([4 * (q + k) + 2 for k in range(4)]), np.stack([sh2[q + k] for k in range(4)]))
        assert np.array_equal(got.view(np.uint32), Q[vx[4 * q + 2]].view(np.uint32)), (name, mode, d, "centres")
        # midpoints of the parent edges, at the owner of each pair
        tw0 = tw[4 * f]
        own = (e0 & 1) == 0
        o = f[own]
        bnd1 = tw0[own] < 0
        sa, sx = sharp(e0[own]), sharp(e0[own] ^ 1)
        vp1 = np.where(bnd1, f32(2), f32(4)).astype(f32)
        av1 = (sa + sx).astype(f32)
        cp1 = (_fsign(sa) + _fsign(sx)).astype(f32)
        pM = P[vx[4 * o + 1]]
        a1 = _rule(pM, Fp[o], Ep[e1[own]], Ep[e0[own]], vp1, cp1, av1, bnd1, _fsign(sharp(e1[own])), _fsign(sa),
                   creased)
        a2 = sh3[nxt[own]]
        tn = tw0[own] >> 2
        t = _qprev(tn)
        eB1 = e1[own] - o + t
        k = o.size
        z3, zk, nk = np.zeros((k, 3), f32), np.zeros(k, f32), np.zeros(k, bool)
        ts = np.where(bnd1, 0, t)
        tns = np.where(bnd1, 0, tn)
        eBs = np.where(bnd1, 0, eB1)
        b1 = _rule(pM, Fp[ts], Ep[eBs], z3, vp1, cp1, av1, nk, _fsign(sharp(eBs)), zk, creased)
        b2 = _rule(pM, Fp[tns], Ep[e0[own]], z3, vp1, cp1, av1, nk, _fsign(sa), zk, creased)
        ids_a = np.stack([4 * o + 1, 4 * nxt[own] + 3])
        pair = _sum_sorted(ids_a, np.stack([a1, a2]))
        quad4 = _sum_sorted(np.concatenate([ids_a, np.stack([4 * t + 1, 4 * tn + 3])]),
                            np.stack([a1, a2, b1, b2]))
        got = np.where(bnd1[:, None], pair, quad4)
        assert np.array_equal(got.view(np.uint32), Q[vx[4 * o + 1]].view(np.uint32)), (name, mode, d, "midpoints")
