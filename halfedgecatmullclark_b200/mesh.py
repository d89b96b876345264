"""Host-side control cage: the ``cc_Mesh`` record of CatmullClark.h.

The arrays keep the reference's exact memory layout so that a ``cc_Mesh``
struct built over them (``Cage.as_cc_mesh``) can be handed to the CUDA
library's C-ABI (``ccs_Create_cuda``) or to any C code written against the
reference header:

* ``halfedges``  : ``cc_Halfedge`` records, 7 x int32 = 28 B
  (CatmullClark.h:37-45)
* ``creases``    : ``cc_Crease`` records {nextID, prevID, float sharpness},
  12 B (CatmullClark.h:30-34); one crease per cage edge
* ``vertex_points`` : ``cc_VertexPoint`` float32 x 3 (CatmullClark.h:18-21)
* ``uvs``        : ``cc_VertexUv`` float32 x 2 (CatmullClark.h:24-27)
* ``v2h``/``e2h``/``f2h`` : the vertex/edge/face -> halfedge maps
  (CatmullClark.h:63-65)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

HALFEDGE_DTYPE = np.dtype([
    ("twinID", "<i4"), ("nextID", "<i4"), ("prevID", "<i4"), ("faceID", "<i4"),
    ("edgeID", "<i4"), ("vertexID", "<i4"), ("uvID", "<i4"),
])
CREASE_DTYPE = np.dtype([("nextID", "<i4"), ("prevID", "<i4"), ("sharpness", "<f4")])
# cc_Halfedge_SemiRegular (CatmullClark.h:48-55); the 3-word form is the
# CC_DISABLE_UV build of the same record.
SEMIREGULAR_DTYPE = np.dtype([("twinID", "<i4"), ("edgeID", "<i4"), ("vertexID", "<i4"), ("uvID", "<i4")])
SEMIREGULAR_NOUV_DTYPE = np.dtype([("twinID", "<i4"), ("edgeID", "<i4"), ("vertexID", "<i4")])


class cc_Mesh(ctypes.Structure):
    """ctypes mirror of ``cc_Mesh`` (CatmullClark.h:58-71)."""
    _fields_ = [
        ("vertexCount", ctypes.c_int32),
        ("uvCount", ctypes.c_int32),
        ("halfedgeCount", ctypes.c_int32),
        ("edgeCount", ctypes.c_int32),
        ("faceCount", ctypes.c_int32),
        ("vertexToHalfedgeIDs", ctypes.c_void_p),
        ("edgeToHalfedgeIDs", ctypes.c_void_p),
        ("faceToHalfedgeIDs", ctypes.c_void_p),
        ("vertexPoints", ctypes.c_void_p),
        ("uvs", ctypes.c_void_p),
        ("halfedges", ctypes.c_void_p),
        ("creases", ctypes.c_void_p),
    ]


class cc_Subd(ctypes.Structure):
    """ctypes mirror of ``cc_Subd`` (CatmullClark.h:136-142)."""
    _fields_ = [
        ("cage", ctypes.c_void_p),
        ("vertexPoints", ctypes.c_void_p),
        ("halfedges", ctypes.c_void_p),
        ("creases", ctypes.c_void_p),
        ("maxDepth", ctypes.c_int32),
    ]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


@dataclass
class Cage:
    """A halfedge control cage with the reference's array layout."""
    vertex_points: np.ndarray            # (V, 3) float32
    halfedges: np.ndarray                # (H,) HALFEDGE_DTYPE
    creases: np.ndarray                  # (E,) CREASE_DTYPE
    v2h: np.ndarray                      # (V,) int32
    e2h: np.ndarray                      # (E,) int32
    f2h: np.ndarray                      # (F,) int32
    uvs: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.vertex_points = np.ascontiguousarray(self.vertex_points, np.float32).reshape(-1, 3)
        self.uvs = np.ascontiguousarray(self.uvs, np.float32).reshape(-1, 2)
        self.halfedges = np.ascontiguousarray(self.halfedges, HALFEDGE_DTYPE)
        self.creases = np.ascontiguousarray(self.creases, CREASE_DTYPE)
        self.v2h = np.ascontiguousarray(self.v2h, np.int32)
        self.e2h = np.ascontiguousarray(self.e2h, np.int32)
        self.f2h = np.ascontiguousarray(self.f2h, np.int32)

    # counts (CatmullClark.h:399-452)
    @property
    def V(self) -> int:
        return int(self.vertex_points.shape[0])

    @property
    def U(self) -> int:
        return int(self.uvs.shape[0])

    @property
    def H(self) -> int:
        return int(self.halfedges.shape[0])

    @property
    def E(self) -> int:
        return int(self.e2h.shape[0])

    @property
    def F(self) -> int:
        return int(self.f2h.shape[0])

    def as_cc_mesh(self) -> cc_Mesh:
        """A ``cc_Mesh`` struct whose pointers alias this cage's arrays.

        The arrays must stay alive (and unmoved) while the struct is in use;
        the returned struct keeps a reference to this cage.
        """
        m = cc_Mesh(self.V, self.U, self.H, self.E, self.F,
                    _ptr(self.v2h), _ptr(self.e2h), _ptr(self.f2h),
                    _ptr(self.vertex_points), _ptr(self.uvs),
                    _ptr(self.halfedges), _ptr(self.creases))
        m._owner = self  # noqa: SLF001 - keep arrays alive
        return m

    def copy(self) -> "Cage":
        return Cage(self.vertex_points.copy(), self.halfedges.copy(), self.creases.copy(),
                    self.v2h.copy(), self.e2h.copy(), self.f2h.copy(), self.uvs.copy())

    def face_sizes(self) -> np.ndarray:
        return np.bincount(self.halfedges["faceID"], minlength=self.F).astype(np.int32)

    def summary(self) -> dict:
        """Census in the spirit of examples/mesh_info.c:320-353."""
        sizes = self.face_sizes()
        boundary = 2 * self.E - self.H
        sharp = int(np.count_nonzero(self.creases["sharpness"]))
        return {"V": self.V, "U": self.U, "H": self.H, "E": self.E, "F": self.F,
                "non_quads": int(np.count_nonzero(sizes != 4)),
                "boundaries": int(boundary), "creases": sharp - int(boundary)}

    @staticmethod
    def from_cc_mesh(m: cc_Mesh) -> "Cage":
        """Copy a ``cc_Mesh`` living in C memory into numpy arrays."""
        def arr(ptr, n, dtype, shape=None):
            if n == 0 or not ptr:
                return np.zeros(shape if shape else (0,), dtype)
            buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
            a = np.frombuffer(buf, dtype=dtype, count=n).copy()
            return a
        V, U, H, E, F = m.vertexCount, m.uvCount, m.halfedgeCount, m.edgeCount, m.faceCount
        pts = arr(m.vertexPoints, 3 * V, np.float32).reshape(-1, 3)
        uvs = arr(m.uvs, 2 * U, np.float32).reshape(-1, 2)
        return Cage(pts, arr(m.halfedges, H, HALFEDGE_DTYPE), arr(m.creases, E, CREASE_DTYPE),
                    arr(m.vertexToHalfedgeIDs, V, np.int32), arr(m.edgeToHalfedgeIDs, E, np.int32),
                    arr(m.faceToHalfedgeIDs, F, np.int32), uvs)


def cage_of_block(ptr: int) -> "Cage":
    """A ``Cage`` whose arrays are views of a single-block ``cc_Mesh`` made by
    the C library (``ccs_LoadCage_cuda``, ``ccs_BuildCage_cuda``); the block
    is released (``ccs_ReleaseCage_cuda``) with the cage."""
    import weakref

    from . import _native as N
    m = cc_Mesh.from_address(ptr)

    def view(addr, dtype, n):
        dtype = np.dtype(dtype)
        if n == 0 or not addr:
            return np.zeros(0, dtype)
        return np.frombuffer((ctypes.c_char * (n * dtype.itemsize)).from_address(addr), dtype, n)

    V, U, E, F, H = m.vertexCount, m.uvCount, m.edgeCount, m.faceCount, m.halfedgeCount
    cage = Cage(view(m.vertexPoints, np.float32, 3 * V).reshape(-1, 3),
                view(m.halfedges, HALFEDGE_DTYPE, H), view(m.creases, CREASE_DTYPE, E),
                view(m.vertexToHalfedgeIDs, np.int32, V), view(m.edgeToHalfedgeIDs, np.int32, E),
                view(m.faceToHalfedgeIDs, np.int32, F), view(m.uvs, np.float32, 2 * U).reshape(-1, 2))
    weakref.finalize(cage, N.lib().ccs_ReleaseCage_cuda, ptr)
    return cage
