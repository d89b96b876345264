"""Build a halfedge control cage from an indexed polygon mesh.

This reproduces the conventions of the reference's OBJ converter
(examples/obj_to_ccm.c, ``LoadObj`` :666-752) so that cages made here index
their halfedges, edges, vertices and creases exactly as the reference would:

* halfedges are numbered face by face in input order; next/prev cycle inside
  the face (``LoadFaceMappings`` :312-348); ``f2h`` is each face's first
  halfedge;
* twins pair (v0 -> v1) with (v1 -> v0); unpaired halfedges get -1
  (``ComputeTwins`` :142-190);
* an edge is represented by the larger halfedge ID of its pair; edges are
  numbered in increasing order of that ID (``LoadEdgeMappings`` :364-402);
* a vertex maps to its largest outgoing halfedge ID, or, on a boundary, to
  the outgoing halfedge without a twin (``LoadVertexHalfedges`` :417-450);
* creases start as self-links with sharpness 0; ``t crease`` tags set the
  sharpness of every edge joining the two tagged vertices, in tag order
  (``ObjReadCrease`` :538-561); boundary edges are then set to 16
  (``MakeBoundariesSharp`` :265-279); finally crease chains are linked
  through vertices where exactly one other sharp edge meets
  (``ComputeCreaseNeighbors`` :197-253).
* a face written without texture indices gets uvID 0 (``ObjReadFace``
  :461-494).

The builder assumes a manifold input (each directed edge used once, one fan
per vertex), which is what every generator in this package produces.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np

from .mesh import CREASE_DTYPE, HALFEDGE_DTYPE, Cage


def build_cage(points: np.ndarray, faces: Sequence[Sequence[int]],
               uvs: np.ndarray | None = None,
               face_uvs: Sequence[Sequence[int]] | None = None,
               crease_tags: Iterable[tuple[int, int, float]] = ()) -> Cage:
    """Make a cage from 0-based polygon vertex lists (and optional UVs).

    ``crease_tags`` holds (v0, v1, sharpness) triples with 0-based vertex
    IDs, the meaning of the reference's ``t crease 2/1/0 v0 v1 s`` lines.
    """
    points = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    V = points.shape[0]
    sizes = np.fromiter((len(f) for f in faces), np.int64, len(faces))
    if np.any(sizes < 3):
        raise ValueError("cage faces need at least 3 vertices")
    H = int(sizes.sum())
    if H >= 2**31 or V >= 2**31:
        raise ValueError("cage too large for int32 indices")
    F = len(faces)
    begin = np.zeros(F + 1, np.int64)
    np.cumsum(sizes, out=begin[1:])
    fv = np.fromiter((v for f in faces for v in f), np.int64, H)
    if fv.size and (fv.min() < 0 or fv.max() >= V):
        raise ValueError("face vertex index out of range")

    he = np.zeros(H, HALFEDGE_DTYPE)
    face_of = np.repeat(np.arange(F, dtype=np.int64), sizes)
    local = np.arange(H, dtype=np.int64) - begin[face_of]
    n = sizes[face_of]
    nxt = begin[face_of] + np.where(local == n - 1, 0, local + 1)
    prv = begin[face_of] + np.where(local == 0, n - 1, local - 1)
    he["vertexID"] = fv
    he["faceID"] = face_of
    he["nextID"] = nxt
    he["prevID"] = prv
    if face_uvs is not None:
        fu = np.fromiter((u for f in face_uvs for u in f), np.int64, H)
        he["uvID"] = fu
    else:
        he["uvID"] = 0

    # twins: directed-edge hash v0 + V * v1, matched against v1 + V * v0
    v0 = fv
    v1 = fv[nxt]
    key = v0 + np.int64(V) * v1
    order = np.argsort(key, kind="stable")
    skey = key[order]
    if skey.size > 1 and np.any(skey[1:] == skey[:-1]):
        raise ValueError("non-manifold cage: a directed edge is used twice")
    want = v1 + np.int64(V) * v0
    pos = np.searchsorted(skey, want)
    pos_c = np.minimum(pos, H - 1)
    found = skey[pos_c] == want
    twin = np.where(found, order[pos_c], -1).astype(np.int64)
    he["twinID"] = twin

    # edges: one bit per halfedge that carries its pair's largest ID
    hid = np.arange(H, dtype=np.int64)
    bits = (hid > twin).astype(np.int64)
    prefix = np.zeros(H + 1, np.int64)
    np.cumsum(bits, out=prefix[1:])
    E = int(prefix[-1])
    he["edgeID"] = prefix[np.maximum(hid, twin)]
    e2h = np.nonzero(bits)[0].astype(np.int32)

    # vertex -> halfedge
    v2h = np.full(V, -1, np.int64)
    np.maximum.at(v2h, fv, hid)
    bnd = twin < 0
    v2h[fv[bnd]] = hid[bnd]

    # creases
    cr = np.zeros(E, CREASE_DTYPE)
    cr["nextID"] = np.arange(E)
    cr["prevID"] = np.arange(E)
    ev0 = fv[e2h]
    ev1 = fv[nxt[e2h]]
    tags = list(crease_tags)
    if tags:
        lut: dict[tuple[int, int], list[int]] = {}
        lo = np.minimum(ev0, ev1)
        hi = np.maximum(ev0, ev1)
        for e, (a, b) in enumerate(zip(lo.tolist(), hi.tolist())):
            lut.setdefault((a, b), []).append(e)
        sharp = cr["sharpness"]
        for a, b, s in tags:
            a, b = int(a), int(b)
            s32 = np.float32(s)
            if a == b:
                hit = np.nonzero((ev0 == a) & (ev1 == a))[0]
                sharp[hit] = s32
            else:
                for e in lut.get((min(a, b), max(a, b)), ()):
                    sharp[e] = s32
    cr["sharpness"][twin[e2h] < 0] = np.float32(16.0)

    cage = Cage(points, he, cr, v2h.astype(np.int32), e2h, begin[:-1].astype(np.int32),
                np.zeros((0, 2), np.float32) if uvs is None else uvs)
    _link_creases(cage)
    return cage


def _link_creases(cage: Cage) -> None:
    """Crease chain links (examples/obj_to_ccm.c:197-253)."""
    he = cage.halfedges
    twin = he["twinID"].astype(np.int64)
    nxt = he["nextID"].astype(np.int64)
    edge = he["edgeID"].astype(np.int64)
    sharp = cage.creases["sharpness"]
    tw = twin.tolist()
    nx = nxt.tolist()
    ed = edge.tolist()
    sh = sharp.tolist()
    e2h = cage.e2h.tolist()

    def next_vertex_he(h):
        t = tw[h]
        return nx[t] if t >= 0 else -1

    new_prev = {}
    new_next = {}
    for e in np.nonzero(sharp > 0.0)[0].tolist():
        h = e2h[e]
        n = nx[h]
        count, cid = 0, -1
        it = next_vertex_he(h)
        while it != h and it >= 0:
            if sh[ed[it]] > 0.0:
                cid = ed[it]
                count += 1
            it = next_vertex_he(it)
        if count == 1 and it == h:
            new_prev[e] = cid
        count, cid = 0, -1
        if sh[ed[n]] > 0.0:
            cid = ed[n]
            count += 1
        it = next_vertex_he(n)
        while it != n and it >= 0:
            if sh[ed[it]] > 0.0 and tw[it] != h:
                cid = ed[it]
                count += 1
            it = next_vertex_he(it)
        if count == 1 and it == n:
            new_next[e] = cid
    for e, p in new_prev.items():
        cage.creases["prevID"][e] = p
    for e, q in new_next.items():
        cage.creases["nextID"][e] = q


def obj_text(points: np.ndarray, faces: Sequence[Sequence[int]],
             uvs: np.ndarray | None = None, face_uvs: Sequence[Sequence[int]] | None = None,
             crease_tags: Iterable[tuple[int, int, float]] = ()) -> str:
    """The OBJ text that the reference's ``LoadObj`` turns into the same cage.

    Floats are written with 9 significant digits so that they parse back to
    the same float32 values.
    """
    out = []
    for p in np.asarray(points, np.float32):
        out.append("v %.9g %.9g %.9g" % (p[0], p[1], p[2]))
    if uvs is not None:
        for t in np.asarray(uvs, np.float32):
            out.append("vt %.9g %.9g" % (t[0], t[1]))
    for k, f in enumerate(faces):
        if face_uvs is not None:
            out.append("f " + " ".join("%d/%d" % (v + 1, t + 1) for v, t in zip(f, face_uvs[k])))
        else:
            out.append("f " + " ".join(str(v + 1) for v in f))
    for a, b, s in crease_tags:
        out.append("t crease 2/1/0 %d %d %.9g" % (a, b, np.float32(s)))
    return "\n".join(out) + "\n"


class _PolygonMesh(ctypes.Structure):
    """ctypes mirror of ``ccs_PolygonMesh`` (include/ccs_cuda.h)."""
    _fields_ = [("vertexCount", ctypes.c_int32), ("uvCount", ctypes.c_int32),
                ("faceCount", ctypes.c_int32), ("creaseTagCount", ctypes.c_int32),
                ("faceOffsets", ctypes.c_void_p), ("faceVertices", ctypes.c_void_p),
                ("faceUvs", ctypes.c_void_p), ("vertexPoints", ctypes.c_void_p),
                ("uvs", ctypes.c_void_p), ("creaseVertices", ctypes.c_void_p),
                ("creaseSharpness", ctypes.c_void_p)]


def build_cage_device(points: np.ndarray, faces: Sequence[Sequence[int]] | None = None,
                      uvs: np.ndarray | None = None,
                      face_uvs: Sequence[Sequence[int]] | None = None,
                      crease_tags: Iterable[tuple[int, int, float]] = (),
                      offsets: np.ndarray | None = None, corners: np.ndarray | None = None,
                      corner_uvs: np.ndarray | None = None, stream=None) -> Cage:
    """``build_cage`` on the GPU (``ccs_BuildCage_cuda``): the same cage, byte
    for byte, with arrays in one page-locked block.

    Faces come either as vertex lists (``faces``, ``face_uvs``) or flattened
    (``offsets`` of length F + 1 and ``corners`` / ``corner_uvs``).  Raises
    ``ValueError`` where the library refuses the input (a face with fewer than
    3 corners or two consecutive corners on one vertex, an index out of
    range, a directed edge used twice).
    """
    from . import _native as N
    from .mesh import cage_of_block

    points = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    if offsets is None:
        sizes = np.fromiter((len(f) for f in faces), np.int64, len(faces))
        offsets = np.zeros(len(faces) + 1, np.int64)
        np.cumsum(sizes, out=offsets[1:])
        corners = np.fromiter((v for f in faces for v in f), np.int64, int(offsets[-1]))
        if face_uvs is not None:
            corner_uvs = np.fromiter((u for f in face_uvs for u in f), np.int64, int(offsets[-1]))
    if int(offsets[-1]) >= 2**31:
        raise ValueError("cage too large for int32 indices")
    off = np.ascontiguousarray(offsets, np.int32)
    fv = np.ascontiguousarray(corners, np.int32)
    fu = None if corner_uvs is None else np.ascontiguousarray(corner_uvs, np.int32)
    uv = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
    tags = list(crease_tags)
    tv = np.ascontiguousarray([(int(a), int(b)) for a, b, _ in tags], np.int32).reshape(-1, 2)
    ts = np.ascontiguousarray([s for _, _, s in tags], np.float32)
    m = _PolygonMesh(points.shape[0], 0 if uv is None else uv.shape[0], off.shape[0] - 1, len(tags),
                     off.ctypes.data, fv.ctypes.data, None if fu is None else fu.ctypes.data,
                     points.ctypes.data, None if uv is None or uv.size == 0 else uv.ctypes.data,
                     tv.ctypes.data if len(tags) else None, ts.ctypes.data if len(tags) else None)
    out = ctypes.c_void_p()
    handle = getattr(stream, "cuda_stream", stream)
    code = N.lib().ccs_BuildCage_cuda(ctypes.byref(m), ctypes.byref(out),
                                      ctypes.c_void_p(int(handle) if handle else 0))
    if code == -1:
        raise ValueError("ccs_BuildCage_cuda refused the polygon mesh")
    N.check(code, "ccs_BuildCage_cuda")
    return cage_of_block(out.value)
