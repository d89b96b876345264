"""Python host mirror of the reference's subdivision API over the C ABI.

``Subd`` wraps one ``cc_Subd`` created by ``ccs_Create_cuda``; its methods
carry the reference's entry-point names (CatmullClark.h:145-212) and raise
``CcsError`` where the C ABI returns a non-zero status.  Results are read
either from the host arrays after ``download()`` (the reference's layout,
byte for byte) or, without a copy, from the device arrays as torch tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .mesh import CREASE_DTYPE, Cage


class _CudaArray:
    """Minimal ``__cuda_array_interface__`` over a device pointer."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None, "stream": None}


def level_counts(cage: Cage, depth: int) -> list[dict]:
    """Counts and array offsets of depths 0..depth (int32-overflow checked)."""
    L = N.lib()
    m = cage.as_cc_mesh()
    out = (N.LevelCounts * (depth + 1))()
    N.check(L.ccs_LevelCounts_cuda(ctypes.byref(m), depth, out), "ccs_LevelCounts_cuda")
    return [{k: int(getattr(o, k)) for k, _ in N.LevelCounts._fields_} for o in out]


def max_supported_depth(cage: Cage) -> int:
    m = cage.as_cc_mesh()
    return int(N.lib().ccs_MaxSupportedDepth_cuda(ctypes.byref(m)))


def cage_step_matrix(cage: Cage, mode: str = "scatter", transpose: bool = False):
    """The cage step of a point rule as CSR arrays (rowptr, col, w): depth-1
    points = S @ cage points (ccs_CageStepMatrix_cuda; host only).  With
    `transpose`, S^T (the adjoint's cage level)."""
    L = N.lib()
    m = cage.as_cc_mesh()
    rows = ctypes.c_int32()
    nnz = ctypes.c_int64()
    md = N.POINT_MODES[mode]
    N.check(L.ccs_CageStepMatrix_cuda(ctypes.byref(m), md, 1 if transpose else 0, ctypes.byref(rows),
                                      ctypes.byref(nnz), None, None, None, 0), "ccs_CageStepMatrix_cuda")
    rp = np.zeros(rows.value + 1, np.int32)
    col = np.zeros(max(nnz.value, 1), np.int32)
    w = np.zeros(max(nnz.value, 1), np.float32)
    N.check(L.ccs_CageStepMatrix_cuda(ctypes.byref(m), md, 1 if transpose else 0, ctypes.byref(rows),
                                      ctypes.byref(nnz), rp.ctypes.data, col.ctypes.data, w.ctypes.data,
                                      nnz.value), "ccs_CageStepMatrix_cuda")
    return rp, col[:nnz.value], w[:nnz.value]


class Subd:
    """A refined hierarchy living on the GPU (and mirrored on the host)."""

    def __init__(self, cage: Cage, depth: int, flags: int = 0):
        self.L = N.lib()
        self.cage = cage
        self.depth = int(depth)
        self.flags = int(flags)
        self._mesh = cage.as_cc_mesh()
        out = ctypes.c_void_p()
        N.check(self.L.ccs_CreateEx_cuda(ctypes.byref(self._mesh), self.depth, self.flags, ctypes.byref(out)),
                "ccs_CreateEx_cuda")
        self.ptr = out.value
        self.levels = level_counts(cage, self.depth)
        last = self.levels[-1]
        self.cumH = last["cumH"] + last["H"]
        self.cumC = last["cumC"] + last["C"]
        self.cumV = last["cumV"] + last["V"]
        self.record_words = 3 if (self.flags & N.FLAG_NO_UV) else 4

    # -- reference entry points (CatmullClark.h:197-212) ------------------
    def _call(self, name: str) -> None:
        N.check(getattr(self.L, name)(self.ptr), name)

    def refine_scatter(self):
        self._call("ccs_Refine_Scatter_cuda")

    def refine_gather(self):
        self._call("ccs_Refine_Gather_cuda")

    def refine_nocreases_scatter(self):
        self._call("ccs_Refine_NoCreases_Scatter_cuda")

    def refine_nocreases_gather(self):
        self._call("ccs_Refine_NoCreases_Gather_cuda")

    def refine_halfedges(self):
        self._call("ccs_RefineHalfedges_cuda")

    def refine_creases(self):
        self._call("ccs_RefineCreases_cuda")

    def refine_vertex_uvs(self):
        self._call("ccs_RefineVertexUvs_cuda")

    def refine_vertex_points(self, mode: str = "scatter"):
        name = {"scatter": "ccs_RefineVertexPoints_Scatter_cuda",
                "gather": "ccs_RefineVertexPoints_Gather_cuda",
                "nocreases_scatter": "ccs_RefineVertexPoints_NoCreases_Scatter_cuda",
                "nocreases_gather": "ccs_RefineVertexPoints_NoCreases_Gather_cuda"}[mode]
        self._call(name)

    def refine(self, mode: str = "scatter"):
        {"scatter": self.refine_scatter, "gather": self.refine_gather,
         "nocreases_scatter": self.refine_nocreases_scatter,
         "nocreases_gather": self.refine_nocreases_gather}[mode]()

    # -- host <-> device ---------------------------------------------------
    def download(self):
        self._call("ccs_Download_cuda")

    def upload_cage_points(self, points: np.ndarray | None = None):
        if points is None:
            N.check(self.L.ccs_UploadCagePoints_cuda(self.ptr, None), "ccs_UploadCagePoints_cuda")
            return
        p = np.ascontiguousarray(points, np.float32).reshape(self.cage.V, 3)
        N.check(self.L.ccs_UploadCagePoints_cuda(self.ptr, p.ctypes.data), "ccs_UploadCagePoints_cuda")

    def set_stream(self, stream) -> None:
        handle = getattr(stream, "cuda_stream", stream)
        N.check(self.L.ccs_SetStream_cuda(self.ptr, ctypes.c_void_p(int(handle) if handle else 0)),
                "ccs_SetStream_cuda")

    def synchronize(self):
        self._call("ccs_Synchronize_cuda")

    def set_flags(self, flags: int):
        N.check(self.L.ccs_SetFlags_cuda(self.ptr, flags), "ccs_SetFlags_cuda")
        self.flags = flags

    # -- host arrays (valid after download) --------------------------------
    def _host(self):
        class _S(ctypes.Structure):
            _fields_ = [("cage", ctypes.c_void_p), ("vertexPoints", ctypes.c_void_p),
                        ("halfedges", ctypes.c_void_p), ("creases", ctypes.c_void_p),
                        ("maxDepth", ctypes.c_int32)]
        return _S.from_address(self.ptr)

    def halfedges(self) -> np.ndarray:
        """cumH x record_words int32 (twin, edge, vertex[, uv]) copy."""
        s = self._host()
        n = self.cumH * self.record_words
        buf = (ctypes.c_int32 * n).from_address(s.halfedges)
        return np.frombuffer(buf, np.int32, n).reshape(-1, self.record_words).copy()

    def creases(self) -> np.ndarray:
        s = self._host()
        buf = (ctypes.c_char * (12 * self.cumC)).from_address(s.creases)
        return np.frombuffer(buf, CREASE_DTYPE, self.cumC).copy()

    def points(self) -> np.ndarray:
        s = self._host()
        buf = (ctypes.c_float * (3 * self.cumV)).from_address(s.vertexPoints)
        return np.frombuffer(buf, np.float32, 3 * self.cumV).reshape(-1, 3).copy()

    # -- device arrays as torch tensors (no copy) ---------------------------
    def device_arrays(self) -> dict:
        import torch
        d = N.DeviceArrays()
        N.check(self.L.ccs_GetDeviceArrays_cuda(self.ptr, ctypes.byref(d)), "ccs_GetDeviceArrays_cuda")
        rw = d.recordBytes // 4
        return {
            "halfedges": torch.as_tensor(_CudaArray(d.halfedges, (d.halfedgeCount, rw), "<i4"), device="cuda"),
            "creases": torch.as_tensor(_CudaArray(d.creases, (d.creaseCount, 3), "<i4"), device="cuda"),
            "points": torch.as_tensor(_CudaArray(d.vertexPoints, (d.vertexCount, 3), "<f4"), device="cuda"),
            "cage_points": torch.as_tensor(_CudaArray(d.cagePoints, (self.cage.V, 3), "<f4"), device="cuda"),
        }

    def normals(self, smooth: bool = True, points=None, out=None):
        """Per-halfedge normals of the finest level as an (H, 3) float32 CUDA
        tensor (ccs_HalfedgeNormal / ccs_HalfedgeNormal_Fast of
        glsl/CatmullClark_Scatter.glsl:931-960).  `points` = a (cumV, 3) CUDA
        tensor of every depth's points (default: the subd's own).  Runs on
        torch's current stream: after refining on the subd's own stream, call
        ``synchronize()`` (or ``set_stream`` it to torch's) first."""
        import torch
        H = self.levels[-1]["H"]
        if out is None:
            dev = points.device if points is not None else torch.device("cuda", torch.cuda.current_device())
            out = torch.empty((H, 3), dtype=torch.float32, device=dev)
        assert out.is_cuda and out.dtype == torch.float32 and out.is_contiguous() and out.numel() == 3 * H
        pp = None
        if points is not None:
            assert points.is_cuda and points.dtype == torch.float32 and points.is_contiguous()
            assert points.numel() == 3 * self.cumV
            pp = points.data_ptr()
        stream = torch.cuda.current_stream(out.device).cuda_stream
        N.check(self.L.ccs_HalfedgeNormals_cuda(self.ptr, pp, out.data_ptr(), 1 if smooth else 0, stream),
                "ccs_HalfedgeNormals_cuda")
        return out

    def export_obj(self, path: str, depth: int | None = None) -> None:
        """Write one depth (default: the finest; 0 = the cage) as an OBJ file,
        formatted on the GPU (ccs_ExportObj_cuda; ExportToObj of
        examples/subd_cpu.c:22-115, byte for byte)."""
        d = self.depth if depth is None else int(depth)
        N.check(self.L.ccs_ExportObj_cuda(self.ptr, d, path.encode()), "ccs_ExportObj_cuda")

    def level_slice(self, level: int, what: str = "V") -> slice:
        """Rows of depth `level` (1..depth) inside the packed arrays."""
        lv = self.levels[level]
        start = {"V": lv["cumV"], "H": lv["cumH"], "C": lv["cumC"]}[what]
        return slice(start, start + lv[what])

    # -- profiling ---------------------------------------------------------
    def set_profiling(self, on: bool):
        N.check(self.L.ccs_SetProfiling_cuda(self.ptr, 1 if on else 0), "ccs_SetProfiling_cuda")

    def read_profile(self, cap: int = 4096) -> list[dict]:
        out = (N.KernelTime * cap)()
        n = self.L.ccs_ReadProfile_cuda(self.ptr, out, cap)
        if n < 0:
            raise N.CcsError(n, "ccs_ReadProfile_cuda")
        return [{"kernel": N.KERNEL_NAMES[out[i].kernel], "level": out[i].level, "ms": out[i].ms,
                 "units": out[i].units} for i in range(n)]

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "ptr", None):
            self.L.ccs_Release_cuda(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
