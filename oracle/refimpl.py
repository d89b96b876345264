"""ctypes front end of the reference itself, compiled from its sources.

TEST INFRASTRUCTURE ONLY.  ``oracle/Makefile``'s ``ref`` target compiles the
reference's CatmullClark.h together with examples/obj_to_ccm.c (for its
``LoadObj``) into ``oracle/_ref/libccref.so``, and the header with float ->
double into ``oracle/_ref/libccref64.so``.  This module calls their public
entry points (``ccs_Create``, ``ccs_Refine_*``, ``ccm_Load``, ``LoadObj``)
through the unmodified ``cc_Mesh``/``cc_Subd`` ABI.  It is used to pin the
oracle, to generate the golden fixtures, and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libccref.so")
REF64_SO = os.path.join(HERE, "_ref", "libccref64.so")

HALFEDGE_DTYPE = np.dtype([("twinID", "<i4"), ("nextID", "<i4"), ("prevID", "<i4"), ("faceID", "<i4"),
                           ("edgeID", "<i4"), ("vertexID", "<i4"), ("uvID", "<i4")])
CREASE_DTYPE = np.dtype([("nextID", "<i4"), ("prevID", "<i4"), ("sharpness", "<f4")])
CREASE64_DTYPE = np.dtype([("nextID", "<i4"), ("prevID", "<i4"), ("sharpness", "<f8")])


class cc_Mesh(ctypes.Structure):
    _fields_ = [("vertexCount", ctypes.c_int32), ("uvCount", ctypes.c_int32),
                ("halfedgeCount", ctypes.c_int32), ("edgeCount", ctypes.c_int32),
                ("faceCount", ctypes.c_int32),
                ("vertexToHalfedgeIDs", ctypes.c_void_p), ("edgeToHalfedgeIDs", ctypes.c_void_p),
                ("faceToHalfedgeIDs", ctypes.c_void_p), ("vertexPoints", ctypes.c_void_p),
                ("uvs", ctypes.c_void_p), ("halfedges", ctypes.c_void_p), ("creases", ctypes.c_void_p)]


class cc_Subd(ctypes.Structure):
    _fields_ = [("cage", ctypes.c_void_p), ("vertexPoints", ctypes.c_void_p),
                ("halfedges", ctypes.c_void_p), ("creases", ctypes.c_void_p),
                ("maxDepth", ctypes.c_int32)]


def available() -> bool:
    return os.path.exists(REF_SO)


def available64() -> bool:
    return os.path.exists(REF64_SO)


_LIB = {}


def lib(fp64: bool = False) -> ctypes.CDLL:
    key = 8 if fp64 else 4
    if key in _LIB:
        return _LIB[key]
    path = REF64_SO if fp64 else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(path + " (build with `make -C oracle ref`)")
    L = ctypes.CDLL(path)
    P, I = ctypes.c_void_p, ctypes.c_int32
    L.ccs_Create.argtypes = [P, I]
    L.ccs_Create.restype = P
    L.ccs_Release.argtypes = [P]
    L.ccs_Release.restype = None
    for fn in ("ccs_Refine_Scatter", "ccs_Refine_Gather", "ccs_Refine_NoCreases_Scatter",
               "ccs_Refine_NoCreases_Gather", "ccs_RefineVertexPoints_Scatter",
               "ccs_RefineVertexPoints_Gather", "ccs_RefineVertexPoints_NoCreases_Scatter",
               "ccs_RefineVertexPoints_NoCreases_Gather", "ccs_RefineHalfedges",
               "ccs_RefineCreases", "ccs_RefineVertexUvs"):
        getattr(L, fn).argtypes = [P]
        getattr(L, fn).restype = None
    for fn in ("ccs_CumulativeHalfedgeCountAtDepth", "ccs_CumulativeVertexCountAtDepth",
               "ccs_CumulativeCreaseCountAtDepth", "ccs_CumulativeEdgeCountAtDepth",
               "ccs_CumulativeFaceCountAtDepth", "ccm_HalfedgeCountAtDepth",
               "ccm_CreaseCountAtDepth", "ccm_FaceCountAtDepth", "ccm_EdgeCountAtDepth",
               "ccm_VertexCountAtDepth"):
        getattr(L, fn).argtypes = [P, I]
        getattr(L, fn).restype = I
    L.ccm_Load.argtypes = [ctypes.c_char_p]
    L.ccm_Load.restype = P
    L.ccm_Release.argtypes = [P]
    L.ccm_Release.restype = None
    L.ccm_Save.argtypes = [P, ctypes.c_char_p]
    L.ccm_Save.restype = ctypes.c_bool
    if not fp64:
        L.LoadObj.argtypes = [ctypes.c_char_p]
        L.LoadObj.restype = P
        L.ccref_set_threads.argtypes = [ctypes.c_int]
        L.ccref_max_threads.restype = ctypes.c_int
    else:
        L.ccref64_set_threads.argtypes = [ctypes.c_int]
    _LIB[key] = L
    return L


def set_threads(n: int) -> None:
    lib().ccref_set_threads(int(n))
    if available64():
        lib(True).ccref64_set_threads(int(n))


def max_threads() -> int:
    return int(lib().ccref_max_threads())


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype)
    dt = np.dtype(dtype)
    buf = (ctypes.c_char * (n * dt.itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dt, count=n).copy()


def mesh_to_arrays(mptr: int) -> dict:
    m = cc_Mesh.from_address(mptr)
    V, U, H, E, F = m.vertexCount, m.uvCount, m.halfedgeCount, m.edgeCount, m.faceCount
    return {
        "points": _arr(m.vertexPoints, 3 * V, np.float32).reshape(-1, 3),
        "uvs": _arr(m.uvs, 2 * U, np.float32).reshape(-1, 2),
        "halfedges": _arr(m.halfedges, H, HALFEDGE_DTYPE),
        "creases": _arr(m.creases, E, CREASE_DTYPE),
        "v2h": _arr(m.vertexToHalfedgeIDs, V, np.int32),
        "e2h": _arr(m.edgeToHalfedgeIDs, E, np.int32),
        "f2h": _arr(m.faceToHalfedgeIDs, F, np.int32),
    }


def load_ccm(path: str) -> dict | None:
    L = lib()
    p = L.ccm_Load(path.encode())
    if not p:
        return None
    try:
        return mesh_to_arrays(p)
    finally:
        L.ccm_Release(p)


def load_obj_text(text: str) -> dict | None:
    """Run the reference's LoadObj (examples/obj_to_ccm.c:666) on OBJ text."""
    L = lib()
    with tempfile.NamedTemporaryFile("w", suffix=".obj", delete=False) as fh:
        fh.write(text)
        name = fh.name
    try:
        p = L.LoadObj(name.encode())
        if not p:
            return None
        try:
            return mesh_to_arrays(p)
        finally:
            L.ccm_Release(p)
    finally:
        os.unlink(name)


class RefCage:
    """A cage as the reference's own ``LoadObj`` builds it (the attributes
    ``RefSubd`` reads), with no code of the CUDA package involved."""

    def __init__(self, arrays: dict):
        self.vertex_points = arrays["points"]
        self.uvs = arrays["uvs"]
        self.halfedges = arrays["halfedges"]
        self.creases = arrays["creases"]
        self.v2h, self.e2h, self.f2h = arrays["v2h"], arrays["e2h"], arrays["f2h"]
        self.V, self.U = len(self.vertex_points), len(self.uvs)
        self.H, self.E, self.F = len(self.halfedges), len(self.creases), len(self.f2h)


def cage_from_obj_text(text: str) -> RefCage:
    """The reference's LoadObj (examples/obj_to_ccm.c:666) on OBJ text."""
    arrays = load_obj_text(text)
    if arrays is None:
        raise ValueError("the reference's LoadObj refused the OBJ text")
    return RefCage(arrays)


class _MeshRef:
    def __init__(self, cage, fp64=False):
        self.keep = []
        if fp64:
            pts = np.ascontiguousarray(cage.vertex_points, np.float64)
            uvs = np.ascontiguousarray(cage.uvs, np.float64)
            cr = np.zeros(cage.E, CREASE64_DTYPE)
            cr["nextID"] = cage.creases["nextID"]
            cr["prevID"] = cage.creases["prevID"]
            cr["sharpness"] = cage.creases["sharpness"]
        else:
            pts = np.ascontiguousarray(cage.vertex_points, np.float32)
            uvs = np.ascontiguousarray(cage.uvs, np.float32)
            cr = np.ascontiguousarray(cage.creases, CREASE_DTYPE)
        he = np.ascontiguousarray(cage.halfedges, HALFEDGE_DTYPE)
        self.keep = [pts, uvs, cr, he, cage.v2h, cage.e2h, cage.f2h]

        def p(a):
            return a.ctypes.data if a.size else None
        self.m = cc_Mesh(cage.V, cage.U, cage.H, cage.E, cage.F, p(cage.v2h), p(cage.e2h),
                         p(cage.f2h), p(pts), p(uvs), p(he), p(cr))


_ENTRY = {
    "scatter": "ccs_Refine_Scatter",
    "gather": "ccs_Refine_Gather",
    "nocreases_scatter": "ccs_Refine_NoCreases_Scatter",
    "nocreases_gather": "ccs_Refine_NoCreases_Gather",
}


class RefSubd:
    """A reference ``cc_Subd`` created by ``ccs_Create`` on a given cage."""

    def __init__(self, cage, depth: int, fp64: bool = False):
        self.L = lib(fp64)
        self.fp64 = fp64
        self.mesh = _MeshRef(cage, fp64)
        self.cage = cage
        self.depth = depth
        self.ptr = self.L.ccs_Create(ctypes.addressof(self.mesh.m), depth)
        if not self.ptr:
            raise MemoryError("ccs_Create failed")
        self.s = cc_Subd.from_address(self.ptr)
        L = self.L
        m = ctypes.addressof(self.mesh.m)
        self.cumH = L.ccs_CumulativeHalfedgeCountAtDepth(m, depth)
        self.cumC = L.ccs_CumulativeCreaseCountAtDepth(m, depth)
        self.cumV = L.ccs_CumulativeVertexCountAtDepth(m, depth)

    def call(self, fn: str) -> None:
        getattr(self.L, fn)(self.ptr)

    def refine(self, mode: str = "scatter") -> None:
        self.call(_ENTRY[mode])

    def halfedges(self) -> np.ndarray:
        return _arr(self.s.halfedges, 4 * self.cumH, np.int32).reshape(-1, 4)

    def creases(self) -> np.ndarray:
        return _arr(self.s.creases, self.cumC, CREASE64_DTYPE if self.fp64 else CREASE_DTYPE)

    def points(self) -> np.ndarray:
        return _arr(self.s.vertexPoints, 3 * self.cumV,
                    np.float64 if self.fp64 else np.float32).reshape(-1, 3)

    def views(self) -> dict:
        """Zero-copy numpy views of the subd's packed arrays (valid until
        close()): halfedges cumH x 4 int32, creases cumC x 3 int32 (the
        sharpness as its bits; FP32 build only), points cumV x 3."""
        def view(ptr, n, dtype):
            dt = np.dtype(dtype)
            return np.frombuffer((ctypes.c_char * (n * dt.itemsize)).from_address(ptr), dtype=dt, count=n)
        out = {"halfedges": view(self.s.halfedges, 4 * self.cumH, np.int32).reshape(-1, 4),
               "points": view(self.s.vertexPoints, 3 * self.cumV,
                              np.float64 if self.fp64 else np.float32).reshape(-1, 3)}
        if not self.fp64:
            out["creases"] = view(self.s.creases, 3 * self.cumC, np.int32).reshape(-1, 3)
        return out

    def close(self) -> None:
        if self.ptr:
            self.L.ccs_Release(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refine(cage, depth: int, mode: str = "scatter", fp64: bool = False):
    s = RefSubd(cage, depth, fp64)
    try:
        s.refine(mode)
        return s.halfedges(), s.creases(), s.points()
    finally:
        s.close()


EXPORT_SO = os.path.join(HERE, "_ref", "libccexport.so")
EXPORT_NOUV_SO = os.path.join(HERE, "_ref", "libccexport_nouv.so")


def export_available() -> bool:
    return os.path.exists(EXPORT_SO) and os.path.exists(EXPORT_NOUV_SO)


def export_obj(cage, depth: int, max_depth: int, halfedges, points, path: str, uv: bool = True) -> None:
    """The reference's ExportToObj (examples/subd_cpu.c:22-115) on a subd
    whose packed arrays are `halfedges` (16-byte records with `uv`, else 12)
    and `points`, over `cage` (a halfedgecatmullclark_b200 Cage)."""
    so = EXPORT_SO if uv else EXPORT_NOUV_SO
    L = ctypes.CDLL(so)
    L.ccref_export_obj.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_char_p]
    L.ccref_export_obj.restype = None
    m = cage.as_cc_mesh()
    he = np.ascontiguousarray(halfedges, np.int32)
    pts = np.ascontiguousarray(points, np.float32)
    s = cc_Subd(ctypes.addressof(m), pts.ctypes.data, he.ctypes.data, None, max_depth)
    L.ccref_export_obj(ctypes.byref(s), depth, path.encode())
