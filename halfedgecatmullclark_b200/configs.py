"""Seeded synthetic cages for the five workloads this library is measured on.

Every generator returns a ``Workload``: the cage (built by ``build_cage``,
i.e. with the reference OBJ converter's conventions), the refinement depth,
and the polygon soup it came from (so that tests can hand the same OBJ text
to the reference's own converter).

1. ``torus_quads``      quad torus 32x16, R=1, r=0.3, jitter sigma 0.01,
                        no creases, no UVs, depth 4.
2. ``mixed_torus``      64x64 grid-torus; 15% of quads split into two
                        triangles; 5% of the split quads give one triangle to
                        an unsplit neighbour quad, forming a pentagon
                        (valences 3-7); an open boundary strip (32 faces of
                        one row removed, boundary edges become sharpness 16);
                        about 10% of edges in crease chains with sharpness
                        U[0,3] per chain; per-corner UVs from the grid
                        parameterisation; depth 6.
3. ``height_grid``      256x256 open quad grid, 20% of quads split along a
                        diagonal, z = 0.1 * sum of 8 random sinusoids, 2% of
                        edges creased with sharpness U[0.5,5]; depth 5.
4. ``fitting_cage``     about 2000 faces generated like (2) on a 44x40
                        torus, depth 5 (the cage-fitting workload).
5. ``batch_cages``      many cages, face counts log-uniform, mixed
                        tri/quad/pentagon, 0-10% crease edges with sharpness
                        U[0,4], depths uniform in a range.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .cage import build_cage, obj_text
from .mesh import Cage


@dataclass
class Workload:
    name: str
    cage: Cage
    depth: int
    points: np.ndarray
    faces: list
    uvs: np.ndarray | None = None
    face_uvs: list | None = None
    crease_tags: list = field(default_factory=list)
    notes: dict = field(default_factory=dict)

    def obj(self) -> str:
        return obj_text(self.points, self.faces, self.uvs, self.face_uvs, self.crease_tags)


def _torus_points(nu: int, nv: int, R: float, r: float) -> np.ndarray:
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    u = 2.0 * np.pi * i / nu
    v = 2.0 * np.pi * j / nv
    x = (R + r * np.cos(v)) * np.cos(u)
    y = (R + r * np.cos(v)) * np.sin(u)
    z = r * np.sin(v)
    return np.stack([x, y, z], -1).reshape(-1, 3)


def torus_quads(nu: int = 32, nv: int = 16, depth: int = 4, seed: int = 0) -> Workload:
    """Workload 1: plain quad torus (512 quads for 32x16)."""
    rng = np.random.default_rng(seed)
    pts = _torus_points(nu, nv, 1.0, 0.3) + rng.normal(0.0, 0.01, (nu * nv, 3))
    pts = pts.astype(np.float32)

    def vid(i, j):
        return (i % nu) * nv + (j % nv)
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)]
             for i in range(nu) for j in range(nv)]
    cage = build_cage(pts, faces)
    return Workload("torus_quads", cage, depth, pts, faces)


def _mixed_grid(nu, nv, rng, wrap_u, wrap_v, split_frac, pent_frac, strip, crease_frac,
                smax, smin=0.0, chains=True, with_uv=True, height=None, torus=(1.0, 0.35)):
    """Grid of nu x nv quads with splits, pentagon merges and crease tags."""
    nvu = nu if wrap_u else nu + 1
    nvv = nv if wrap_v else nv + 1

    def vid(i, j):
        return (i % nvu if wrap_u else i) * nvv + (j % nvv if wrap_v else j)

    if height is None:
        pts = _torus_points(nvu, nvv, *torus)
    else:
        i, j = np.meshgrid(np.arange(nvu), np.arange(nvv), indexing="ij")
        x = i / nu
        y = j / nv
        pts = np.stack([x, y, height(x, y)], -1).reshape(-1, 3)
    pts = pts.astype(np.float32)

    alive = np.ones((nu, nv), bool)
    if strip:
        alive[:strip, 0] = False
    cells = np.argwhere(alive)
    nsplit = int(round(split_frac * len(cells)))
    split_cells = cells[rng.choice(len(cells), nsplit, replace=False)] if nsplit else np.zeros((0, 2), int)
    split = {}
    for (i, j) in split_cells.tolist():
        split[(i, j)] = int(rng.integers(2))  # 0: diagonal a-c, 1: diagonal b-d

    faces = []
    face_uv_keys = []

    def corners(i, j):
        return [(i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)]

    # pentagon merges: a split quad hands one triangle to an unsplit neighbour
    merged_into = {}
    used = set()
    if pent_frac > 0 and split:
        keys = list(split.keys())
        rng.shuffle(keys)
        target = int(round(pent_frac * len(keys)))
        for (i, j) in keys:
            if len(merged_into) >= target:
                break
            if (i, j) in used:
                continue
            d = split[(i, j)]
            # with diagonal a-c the triangles are (a,b,c) and (a,c,d); the
            # first owns grid edges a-b (below) and b-c (right)
            options = [((i, j - 1), 0, "below"), ((i + 1, j), 0, "right"),
                       ((i, j + 1), 1, "above"), ((i - 1, j), 1, "left")] if d == 0 else \
                      [((i, j - 1), 0, "below"), ((i - 1, j), 0, "left"),
                       ((i + 1, j), 1, "right"), ((i, j + 1), 1, "above")]
            rng.shuffle(options)
            for (ni, nj), tri, side in options:
                ni2 = ni % nu if wrap_u else ni
                nj2 = nj % nv if wrap_v else nj
                if not (0 <= ni2 < nu and 0 <= nj2 < nv):
                    continue
                if not alive[ni2, nj2] or (ni2, nj2) in split or (ni2, nj2) in used:
                    continue
                merged_into[(i, j)] = (tri, (ni2, nj2), side)
                used.add((i, j))
                used.add((ni2, nj2))
                break

    def tri_corners(i, j, d, t):
        a, b, c, dd = corners(i, j)
        if d == 0:
            return [a, b, c] if t == 0 else [a, c, dd]
        return [a, b, dd] if t == 0 else [b, c, dd]

    def merge(quad, tri):
        # merge two faces (corner lists) sharing exactly one edge
        qs = [(x % nvu if wrap_u else x, y % nvv if wrap_v else y) for x, y in quad]
        ts = [(x % nvu if wrap_u else x, y % nvv if wrap_v else y) for x, y in tri]
        for k in range(len(qs)):
            a, b = qs[k], qs[(k + 1) % len(qs)]
            for m in range(len(ts)):
                if ts[m] == b and ts[(m + 1) % len(ts)] == a:
                    # walk quad from b around to a, then tri's remaining
                    # vertex, moved into the quad's unwrapped frame
                    qrot = [quad[(k + 1 + s) % len(quad)] for s in range(len(quad))]
                    qb, tb = quad[(k + 1) % len(quad)], tri[m]
                    ox, oy = qb[0] - tb[0], qb[1] - tb[1]
                    extra = [(tri[(m + 2 + s) % len(tri)][0] + ox, tri[(m + 2 + s) % len(tri)][1] + oy)
                             for s in range(len(tri) - 2)]
                    return qrot + extra
        raise RuntimeError("faces do not share an edge")

    pent_quad = {v[1]: (k, v[0]) for k, v in merged_into.items()}
    for i in range(nu):
        for j in range(nv):
            if not alive[i, j]:
                continue
            if (i, j) in split:
                d = split[(i, j)]
                for t in (0, 1):
                    if (i, j) in merged_into and merged_into[(i, j)][0] == t:
                        continue
                    faces.append(tri_corners(i, j, d, t))
            elif (i, j) in pent_quad:
                (si, sj), t = pent_quad[(i, j)]
                faces.append(merge(corners(i, j), tri_corners(si, sj, split[(si, sj)], t)))
            else:
                faces.append(corners(i, j))

    # UVs: one entry per unwrapped grid corner, (i/nu, j/nv) in [0,1]
    uv_index = {}
    uvs = []
    face_uvs = []
    vfaces = []
    for f in faces:
        vf = []
        uf = []
        for (x, y) in f:
            vf.append(vid(x, y))
            if (x, y) not in uv_index:
                uv_index[(x, y)] = len(uvs)
                uvs.append((x / nu, y / nv))
            uf.append(uv_index[(x, y)])
        vfaces.append(vf)
        face_uvs.append(uf)

    # crease chains along grid lines (or single edges when chains=False)
    edges = set()
    for f in vfaces:
        for k in range(len(f)):
            a, b = f[k], f[(k + 1) % len(f)]
            edges.add((min(a, b), max(a, b)))
    tags = []
    tagged = set()
    target = int(round(crease_frac * len(edges)))
    guard = 0
    while len(tagged) < target and guard < 100 * max(target, 1):
        guard += 1
        s = float(rng.uniform(smin, smax))
        i = int(rng.integers(nvu))
        j = int(rng.integers(nvv))
        if chains:
            du, dv = ((1, 0), (0, 1))[int(rng.integers(2))]
            length = int(rng.integers(3, 12))
        else:
            du, dv = ((1, 0), (0, 1))[int(rng.integers(2))]
            length = 1
        for _ in range(length):
            i2, j2 = i + du, j + dv
            if not wrap_u and i2 >= nvu:
                break
            if not wrap_v and j2 >= nvv:
                break
            a, b = vid(i, j), vid(i2, j2)
            key = (min(a, b), max(a, b))
            if key in edges and key not in tagged:
                tags.append((a, b, s))
                tagged.add(key)
            i, j = i2 % nvu if wrap_u else i2, j2 % nvv if wrap_v else j2
            if len(tagged) >= target:
                break
    uv_arr = np.asarray(uvs, np.float32) if with_uv else None
    return pts, vfaces, uv_arr, (face_uvs if with_uv else None), tags, {
        "splits": len(split), "pentagons": len(merged_into), "crease_edges": len(tagged)}


def mixed_torus(nu: int = 64, nv: int = 64, depth: int = 6, seed: int = 0,
                strip: int = 32, crease_frac: float = 0.10, smax: float = 3.0,
                with_uv: bool = True) -> Workload:
    """Workload 2: mixed-valence torus with creases, UVs and a boundary strip."""
    rng = np.random.default_rng(seed)
    pts, faces, uvs, fuv, tags, notes = _mixed_grid(
        nu, nv, rng, True, True, 0.15, 0.05, strip, crease_frac, smax, with_uv=with_uv)
    cage = build_cage(pts, faces, uvs, fuv, tags)
    return Workload("mixed_torus", cage, depth, pts, faces, uvs, fuv, tags, notes)


def height_grid(n: int = 256, depth: int = 5, seed: int = 0) -> Workload:
    """Workload 3: open height-field grid with diagonal splits and creases."""
    rng = np.random.default_rng(seed)
    freq = rng.uniform(-4.0, 4.0, (8, 2)) * 2.0 * np.pi
    phase = rng.uniform(0.0, 2.0 * np.pi, 8)

    def height(x, y):
        z = np.zeros_like(x, dtype=np.float64)
        for k in range(8):
            z += np.sin(freq[k, 0] * x + freq[k, 1] * y + phase[k])
        return 0.1 * z
    pts, faces, _, _, tags, notes = _mixed_grid(
        n, n, rng, False, False, 0.20, 0.0, 0, 0.02, 5.0, smin=0.5, chains=False,
        with_uv=False, height=height)
    cage = build_cage(pts, faces, None, None, tags)
    return Workload("height_grid", cage, depth, pts, faces, None, None, tags, notes)


def fitting_cage(depth: int = 5, seed: int = 0, nu: int = 44, nv: int = 40) -> Workload:
    """Workload 4: ~2000-face mixed quad/triangle cage."""
    rng = np.random.default_rng(seed)
    pts, faces, uvs, fuv, tags, notes = _mixed_grid(
        nu, nv, rng, True, True, 0.15, 0.0, 0, 0.10, 3.0)
    cage = build_cage(pts, faces, uvs, fuv, tags)
    return Workload("fitting_cage", cage, depth, pts, faces, uvs, fuv, tags, notes)


def batch_cages(count: int = 512, fmin: int = 50, fmax: int = 5000, dmin: int = 2,
                dmax: int = 6, seed: int = 0) -> list[Workload]:
    """Workload 5: many uneven cages (sizes log-uniform, depths uniform)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        target = float(np.exp(rng.uniform(np.log(fmin), np.log(fmax))))
        nu = max(3, int(round(np.sqrt(target * 1.5))))
        nv = max(3, int(round(target / nu / 1.08)))
        depth = int(rng.integers(dmin, dmax + 1))
        frac = float(rng.uniform(0.0, 0.10))
        sub = np.random.default_rng(int(rng.integers(2**31)))
        pts, faces, uvs, fuv, tags, notes = _mixed_grid(
            nu, nv, sub, True, True, 0.15, 0.05, 0, frac, 4.0, with_uv=False)
        cage = build_cage(pts, faces, None, None, tags)
        out.append(Workload("batch_%d" % k, cage, depth, pts, faces, None, None, tags, notes))
    return out


WORKLOADS = {
    "torus_quads": torus_quads,
    "mixed_torus": mixed_torus,
    "height_grid": height_grid,
    "fitting_cage": fitting_cage,
}
