"""ctypes front end of the CPU oracle (oracle/ccs_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product package never
imports this module.

``refine`` runs the full reference pipeline (topology, creases, UVs and
points) sequentially; ``refine_points`` recomputes only the points over a
given topology; ``adjoint`` applies the transposed point rules.  Passing
``real=np.float64`` selects the FP64 oracle (points in double over the FP32
topology and sharpness).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CREASE_DTYPE = np.dtype([("nextID", "<i4"), ("prevID", "<i4"), ("sharpness", "<f4")])


class _Cage(ctypes.Structure):
    _fields_ = [("V", ctypes.c_int32), ("U", ctypes.c_int32), ("H", ctypes.c_int32),
                ("E", ctypes.c_int32), ("F", ctypes.c_int32),
                ("v2h", ctypes.c_void_p), ("e2h", ctypes.c_void_p), ("f2h", ctypes.c_void_p),
                ("he", ctypes.c_void_p), ("cr", ctypes.c_void_p), ("uvs", ctypes.c_void_p)]


class _Subd(ctypes.Structure):
    _fields_ = [("cage", ctypes.c_void_p), ("D", ctypes.c_int32), ("stride", ctypes.c_int32),
                ("he", ctypes.c_void_p), ("cr", ctypes.c_void_p), ("pts", ctypes.c_void_p)]


_LIBS: dict = {}


def _lib(real) -> ctypes.CDLL:
    key = np.dtype(real).itemsize
    if key in _LIBS:
        return _LIBS[key]
    name = "liboracle32.so" if key == 4 else "liboracle64.so"
    path = os.path.join(HERE, name)
    src = os.path.join(HERE, "ccs_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, name], check=True)
    lib = ctypes.CDLL(path)
    P, I = ctypes.c_void_p, ctypes.c_int32
    for fn in ("or_H_at", "or_C_at", "or_F_at", "or_E_at", "or_V_at",
               "or_cumH", "or_cumC", "or_cumE", "or_cumV", "or_cumF"):
        getattr(lib, fn).argtypes = [P, I]
        getattr(lib, fn).restype = I
    for fn in ("or_refine_halfedges", "or_refine_creases", "or_refine_uvs", "or_refine_topology"):
        getattr(lib, fn).argtypes = [P]
        getattr(lib, fn).restype = None
    for fn in ("or_refine_points_scatter", "or_refine_points_gather",
               "or_refine_points_nocreases_scatter", "or_refine_points_nocreases_gather"):
        getattr(lib, fn).argtypes = [P, P]
        getattr(lib, fn).restype = None
    lib.or_step_points_scatter.argtypes = [P, I, I, P]
    lib.or_step_points_scatter.restype = None
    lib.or_adjoint_points_scatter.argtypes = [P, P, P, P]
    lib.or_adjoint_points_scatter.restype = None
    lib.or_edge_to_halfedge.argtypes = [P, I, I]
    lib.or_edge_to_halfedge.restype = I
    lib.or_vertex_to_halfedge.argtypes = [P, I, I]
    lib.or_vertex_to_halfedge.restype = I
    lib.or_real_size.restype = I
    assert lib.or_real_size() == key
    _LIBS[key] = lib
    return lib


def _ptr(a):
    return a.ctypes.data if a is not None and a.size else None


class _CageRef:
    """Keeps a cage's arrays alive behind an oracle cage struct."""

    def __init__(self, cage):
        self.cage = cage
        self.s = _Cage(cage.V, cage.U, cage.H, cage.E, cage.F,
                       _ptr(cage.v2h), _ptr(cage.e2h), _ptr(cage.f2h),
                       _ptr(cage.halfedges), _ptr(cage.creases), _ptr(cage.uvs))

    @property
    def addr(self):
        return ctypes.addressof(self.s)


def counts(cage, depth: int) -> dict:
    """Per-level and cumulative counts from the reference's int32 formulas."""
    lib = _lib(np.float32)
    c = _CageRef(cage)
    out = {}
    for key, fn in (("H", "or_H_at"), ("C", "or_C_at"), ("F", "or_F_at"), ("E", "or_E_at"),
                    ("V", "or_V_at"), ("cumH", "or_cumH"), ("cumC", "or_cumC"),
                    ("cumE", "or_cumE"), ("cumV", "or_cumV"), ("cumF", "or_cumF")):
        out[key] = [int(getattr(lib, fn)(c.addr, d)) for d in range(depth + 1)]
    return out


def edge_to_halfedge(cage, edge: int, depth: int) -> int:
    c = _CageRef(cage)
    return int(_lib(np.float32).or_edge_to_halfedge(c.addr, edge, depth))


def vertex_to_halfedge(cage, vertex: int, depth: int) -> int:
    c = _CageRef(cage)
    return int(_lib(np.float32).or_vertex_to_halfedge(c.addr, vertex, depth))


_POINT_FNS = {
    "scatter": "or_refine_points_scatter",
    "gather": "or_refine_points_gather",
    "nocreases_scatter": "or_refine_points_nocreases_scatter",
    "nocreases_gather": "or_refine_points_nocreases_gather",
}


def refine_topology(cage, depth: int, stride: int = 4):
    """Halfedges (sum_H x stride int32) and creases of levels 1..depth."""
    cnt = counts(cage, depth)
    he = np.zeros((cnt["cumH"][depth], stride), np.int32)
    cr = np.zeros(cnt["cumC"][depth], CREASE_DTYPE)
    c = _CageRef(cage)
    s = _Subd(c.addr, depth, stride, _ptr(he), _ptr(cr), None)
    _lib(np.float32).or_refine_topology(ctypes.addressof(s))
    return he, cr


def refine_points(cage, depth: int, he, cr, mode: str = "scatter", real=np.float32,
                  cage_points=None, stride: int = 4):
    """Points (sum_V x 3) of levels 1..depth over a given topology."""
    cnt = counts(cage, depth)
    pts = np.zeros((cnt["cumV"][depth], 3), real)
    cp = np.ascontiguousarray(cage.vertex_points if cage_points is None else cage_points, real)
    he = np.ascontiguousarray(he, np.int32)
    cr = np.ascontiguousarray(cr, CREASE_DTYPE)
    c = _CageRef(cage)
    s = _Subd(c.addr, depth, stride, _ptr(he), _ptr(cr), _ptr(pts))
    getattr(_lib(real), _POINT_FNS[mode])(ctypes.addressof(s), _ptr(cp))
    return pts


def step_points(cage, depth: int, he, cr, pts, d: int, creased: bool = True, cage_points=None,
                stride: int = 4):
    """Level d+1 of `pts` (sum_V x 3, levels 1..depth, FP32) recomputed by the
    scatter rules from the level-d rows already in `pts` (d = 0: the cage
    points): returns a copy of `pts` with only level d+1 replaced."""
    out = np.array(pts, np.float32, copy=True, order="C")
    cp = np.ascontiguousarray(cage.vertex_points if cage_points is None else cage_points, np.float32)
    he = np.ascontiguousarray(he, np.int32)
    cr = np.ascontiguousarray(cr, CREASE_DTYPE)
    c = _CageRef(cage)
    s = _Subd(c.addr, depth, stride, _ptr(he), _ptr(cr), _ptr(out))
    _lib(np.float32).or_step_points_scatter(ctypes.addressof(s), d, 1 if creased else 0, _ptr(cp))
    return out


def refine(cage, depth: int, mode: str = "scatter", real=np.float32, stride: int = 4,
           cage_points=None):
    he, cr = refine_topology(cage, depth, stride)
    pts = refine_points(cage, depth, he, cr, mode, real, cage_points, stride)
    return he, cr, pts


def adjoint(cage, depth: int, he, cr, grad, real=np.float64, stride: int = 4):
    """Cage-point gradient of <grad, points> under the creased scatter rule."""
    cnt = counts(cage, depth)
    grad = np.ascontiguousarray(grad, real).reshape(-1, 3)
    assert grad.shape[0] == cnt["cumV"][depth]
    work = np.zeros_like(grad)
    gcage = np.zeros((cage.V, 3), real)
    he = np.ascontiguousarray(he, np.int32)
    cr = np.ascontiguousarray(cr, CREASE_DTYPE)
    c = _CageRef(cage)
    s = _Subd(c.addr, depth, stride, _ptr(he), _ptr(cr), None)
    _lib(real).or_adjoint_points_scatter(ctypes.addressof(s), _ptr(grad), _ptr(work), _ptr(gcage))
    return gcage


def level_slice(cage, depth: int, level: int, what: str = "V"):
    """Row range of level `level` (1..depth) inside the packed arrays."""
    cnt = counts(cage, depth)
    key = {"V": "cumV", "H": "cumH", "C": "cumC"}[what]
    per = {"V": "V", "H": "H", "C": "C"}[what]
    start = cnt[key][level - 1]
    return slice(start, start + cnt[per][level])


def halfedge_normals(he_level, pts_level, smooth: bool = True):
    """Per-halfedge normals of one quad level, in float64.

    Restates glsl/CatmullClark_Scatter.glsl:931-940 (ccs_HalfedgeNormal_Fast:
    normalize(cross(P[v(next h)] - P[v(h)], P[v(prev h)] - P[v(h)]))) and
    :943-960 (ccs_HalfedgeNormal: add the fast normals of the halfedges met
    walking prev-vertex halfedges, twin(prev h), back to h and normalise; a
    walk that meets a boundary returns the fast normal).  `he_level` holds the
    level's records (twin, edge, vertex[, uv]) and `pts_level` its points.
    """
    he = np.asarray(he_level)
    P = np.asarray(pts_level, np.float64)
    H = he.shape[0]
    ids = np.arange(H, dtype=np.int64)
    nxt = (ids & ~3) | ((ids + 1) & 3)
    prv = (ids & ~3) | ((ids - 1) & 3)
    vert = he[:, 2].astype(np.int64)
    twin = he[:, 0].astype(np.int64)

    def unit(v):
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    v0 = P[vert]
    fast = unit(np.cross(P[vert[nxt]] - v0, P[vert[prv]] - v0))
    if not smooth:
        return fast
    acc = np.zeros_like(fast)
    it = twin[prv]                       # ccs_PrevVertexHalfedgeID (CatmullClark.h:1168-1175)
    live = (it >= 0) & (it != ids)
    for _ in range(H):
        if not live.any():
            break
        acc[live] += fast[it[live]]
        step = it.copy()
        step[live] = twin[prv[it[live]]]
        it = np.where(live, step, it)
        live = live & (it >= 0) & (it != ids)
    closed = it >= 0
    out = fast.copy()
    out[closed] = unit(fast[closed] + acc[closed])
    return out


def export_obj_text(cage, depth: int, halfedges=None, points=None, uv: bool = True) -> bytes:
    """The bytes of ExportToObj (examples/subd_cpu.c:22-115) for one depth.

    Depth 0 prints the cage; depth >= 1 the level's rows of the packed
    `halfedges` (twin, edge, vertex[, uv]) and `points`.  Floats print as C's
    "%f" (exact value rounded to 6 decimals, ties to even: Python's "%f" on
    the float64 value of the float32 agrees); texture coordinates at depth
    >= 1 decode the uvID as (x & 0xFFFF) / 65535.0f in float32 (:374-383).
    """
    out = ["# Vertices\n"]
    f6 = lambda x: "%f" % float(x)
    if depth == 0:
        for p in np.asarray(cage.vertex_points, np.float32):
            out.append("v %s %s %s\n" % (f6(p[0]), f6(p[1]), f6(p[2])))
        for t in np.asarray(cage.uvs, np.float32).reshape(-1, 2):
            out.append("vt %s %s\n" % (f6(t[0]), f6(t[1])))
        out.append("\n# Topology\n")
        he = cage.halfedges
        for f in range(cage.F):
            h0 = int(cage.f2h[f])
            corners = [h0]
            h = int(he["nextID"][h0])
            while h != h0:
                corners.append(h)
                h = int(he["nextID"][h])
            out.append("f " + " ".join("%d/%d" % (he["vertexID"][c] + 1, he["uvID"][c] + 1) for c in corners) + "\n")
        return "".join(out).encode()
    hs = level_slice(cage, depth, depth, "H")
    vs = level_slice(cage, depth, depth, "V")
    rec = np.asarray(halfedges)[hs]
    P = np.asarray(points, np.float32)[vs]
    for p in P:
        out.append("v %s %s %s\n" % (f6(p[0]), f6(p[1]), f6(p[2])))
    if uv:
        x = rec[:, 3].astype(np.int64) & 0xFFFFFFFF
        u = (x & 0xFFFF).astype(np.float32) / np.float32(65535.0)
        v = ((x >> 16) & 0xFFFF).astype(np.float32) / np.float32(65535.0)
        for a, b in zip(u, v):
            out.append("vt %s %s\n" % (f6(a), f6(b)))
    out.append("\n# Topology\n")
    vert = rec[:, 2] + 1
    for f in range(rec.shape[0] // 4):
        if uv:
            out.append("f %d/%d %d/%d %d/%d %d/%d\n" % (vert[4 * f], 4 * f + 1, vert[4 * f + 1], 4 * f + 2,
                                                       vert[4 * f + 2], 4 * f + 3, vert[4 * f + 3], 4 * f + 4))
        else:
            out.append("f %d %d %d %d\n" % tuple(vert[4 * f:4 * f + 4]))
    out.append("\n")
    return "".join(out).encode()
