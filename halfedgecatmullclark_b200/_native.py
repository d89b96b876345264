"""ctypes binding of the C ABI in include/ccs_cuda.h (lib/libccs_cuda.so).

There is no fallback: if the CUDA library has not been built, ``lib()``
raises, and every refinement call in this package goes through it.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libccs_cuda.so")

CCS_OK = 0
STATUS = {
    0: "CCS_OK", -1: "CCS_ERR_ARG", -2: "CCS_ERR_ALLOC", -3: "CCS_ERR_OVERFLOW", -4: "CCS_ERR_CUDA",
    -5: "CCS_ERR_TIMEOUT", -6: "CCS_ERR_STATE", -7: "CCS_ERR_UNSUPPORTED", -8: "CCS_ERR_SCRATCH_LIMIT",
}
FLAG_NO_UV = 1 << 0
FLAG_PAGEABLE_HOST = 1 << 1
FLAG_DETERMINISTIC = 1 << 2
FLAG_NO_GRAPH = 1 << 3
FLAG_SEPARATE_PASSES = 1 << 4

POINTS_SCATTER, POINTS_GATHER, POINTS_NOCREASES_SCATTER, POINTS_NOCREASES_GATHER = 0, 1, 2, 3
POINT_MODES = {"scatter": 0, "gather": 1, "nocreases_scatter": 2, "nocreases_gather": 3}

KERNEL_NAMES = ["topology", "creases", "face_points", "edge_points", "vertex_points", "clear",
                "level_fused", "adjoint", "uvs", "level_points", "old_vertices", "ring_stats", "adj_edges",
                "adj_faces", "adj_vertices", "exact_points", "step", "level_step", "level_step_points",
                "adj_step", "crease_stats", "cage_side", "cage_map",
                "adj_cage_map"]


class CcsError(RuntimeError):
    """A non-zero status returned by the C ABI."""

    def __init__(self, code: int, where: str):
        self.code = int(code)
        super().__init__("%s failed: %s (%d)" % (where, STATUS.get(self.code, "?"), self.code))


class DeviceArrays(ctypes.Structure):
    _fields_ = [("halfedges", ctypes.c_void_p), ("creases", ctypes.c_void_p),
                ("vertexPoints", ctypes.c_void_p), ("cagePoints", ctypes.c_void_p),
                ("halfedgeCount", ctypes.c_int64), ("creaseCount", ctypes.c_int64),
                ("vertexCount", ctypes.c_int64), ("recordBytes", ctypes.c_int32)]


class LevelCounts(ctypes.Structure):
    _fields_ = [("H", ctypes.c_int64), ("F", ctypes.c_int64), ("E", ctypes.c_int64),
                ("V", ctypes.c_int64), ("C", ctypes.c_int64),
                ("cumH", ctypes.c_int64), ("cumC", ctypes.c_int64), ("cumV", ctypes.c_int64)]


class BatchArrays(ctypes.Structure):
    _fields_ = [("halfedges", ctypes.c_void_p), ("creases", ctypes.c_void_p), ("points", ctypes.c_void_p),
                ("cagePoints", ctypes.c_void_p), ("gradPoints", ctypes.c_void_p),
                ("gradCagePoints", ctypes.c_void_p), ("halfedgeCount", ctypes.c_int64),
                ("creaseCount", ctypes.c_int64), ("pointCount", ctypes.c_int64),
                ("cagePointCount", ctypes.c_int64)]


class BatchCageInfo(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_int32), ("cagePointOffset", ctypes.c_int64),
                ("cagePointCount", ctypes.c_int64), ("halfedgeOffset", ctypes.c_int64),
                ("halfedgeCount", ctypes.c_int64), ("creaseOffset", ctypes.c_int64),
                ("creaseCount", ctypes.c_int64), ("pointOffset", ctypes.c_int64),
                ("pointCount", ctypes.c_int64), ("finestPointOffset", ctypes.c_int64),
                ("finestPointCount", ctypes.c_int64)]


class KernelTime(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("level", ctypes.c_int32), ("ms", ctypes.c_float),
                ("units", ctypes.c_int64)]


# Every symbol include/ccs_cuda.h declares, with its signature.
_P, _I, _U = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32
SIGNATURES = {
    "ccs_Create_cuda": ([_P, ctypes.c_int32], _P),
    "ccs_CreateEx_cuda": ([_P, ctypes.c_int32, _U, ctypes.POINTER(_P)], _I),
    "ccs_Release_cuda": ([_P], None),
    "ccs_LoadCage_cuda": ([ctypes.c_char_p], _P),
    "ccs_BuildCage_cuda": ([_P, _P, _P], _I),
    "ccs_ReleaseCage_cuda": ([_P], None),
    "ccs_SaveCage_cuda": ([_P, ctypes.c_char_p], _I),
    "ccs_Refine_Scatter_cuda": ([_P], _I),
    "ccs_Refine_Gather_cuda": ([_P], _I),
    "ccs_RefineVertexPoints_Gather_cuda": ([_P], _I),
    "ccs_RefineVertexPoints_Scatter_cuda": ([_P], _I),
    "ccs_RefineHalfedges_cuda": ([_P], _I),
    "ccs_RefineCreases_cuda": ([_P], _I),
    "ccs_RefineVertexUvs_cuda": ([_P], _I),
    "ccs_Refine_NoCreases_Gather_cuda": ([_P], _I),
    "ccs_Refine_NoCreases_Scatter_cuda": ([_P], _I),
    "ccs_RefineVertexPoints_NoCreases_Gather_cuda": ([_P], _I),
    "ccs_RefineVertexPoints_NoCreases_Scatter_cuda": ([_P], _I),
    "ccs_Download_cuda": ([_P], _I),
    "ccs_UploadCagePoints_cuda": ([_P, _P], _I),
    "ccs_SetStream_cuda": ([_P, _P], _I),
    "ccs_GetStream_cuda": ([_P], _P),
    "ccs_Synchronize_cuda": ([_P], _I),
    "ccs_SetFlags_cuda": ([_P, _U], _I),
    "ccs_GetFlags_cuda": ([_P], _U),
    "ccs_GetDeviceArrays_cuda": ([_P, ctypes.POINTER(DeviceArrays)], _I),
    "ccs_RefinePointsDevice_cuda": ([_P, _P, _P, _I, _P], _I),
    "ccs_AdjointPointsDevice_cuda": ([_P, _P, _P, _P], _I),
    "ccs_HalfedgeNormals_cuda": ([_P, _P, _P, ctypes.c_int, _P], _I),
    "ccs_CageStepMatrix_cuda": ([_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                 ctypes.POINTER(ctypes.c_int64), _P, _P, _P, ctypes.c_int64], _I),
    "ccs_ExportObj_cuda": ([_P, ctypes.c_int32, ctypes.c_char_p], _I),
    "ccs_AdjointPointsDeviceNoAlloc_cuda": ([_P, _P, _P, _P], _I),
    "ccs_BatchCreate_cuda": ([_P, _P, ctypes.c_int32, _U, ctypes.POINTER(_P)], _I),
    "ccs_BatchRelease_cuda": ([_P], None),
    "ccs_BatchRefine_cuda": ([_P, _I], _I),
    "ccs_BatchRefinePoints_cuda": ([_P, _I], _I),
    "ccs_BatchAdjointPoints_cuda": ([_P], _I),
    "ccs_BatchAdjointDistance_cuda": ([_P, _P], _I),
    "ccs_BatchGetArrays_cuda": ([_P, ctypes.POINTER(BatchArrays)], _I),
    "ccs_BatchCageInfo_cuda": ([_P, ctypes.c_int32, ctypes.POINTER(BatchCageInfo)], _I),
    "ccs_BatchSetStream_cuda": ([_P, _P], _I),
    "ccs_BatchSetSchedule_cuda": ([_P, ctypes.c_int32], _I),
    "ccs_BatchSetLaunchMode_cuda": ([_P, ctypes.c_int32], _I),
    "ccs_BatchSynchronize_cuda": ([_P], _I),
    "ccs_BatchDownload_cuda": ([_P, ctypes.c_int32, _P], _I),
    "ccs_BarrierTimeoutSelfTest_cuda": ([], _I),
    "ccs_LevelCounts_cuda": ([_P, ctypes.c_int32, ctypes.POINTER(LevelCounts)], _I),
    "ccs_MaxSupportedDepth_cuda": ([_P], ctypes.c_int32),
    "ccs_SetProfiling_cuda": ([_P, _I], _I),
    "ccs_ReadProfile_cuda": ([_P, ctypes.POINTER(KernelTime), _I], _I),
    "ccs_KernelName_cuda": ([_I], ctypes.c_char_p),
    "ccs_LastError_cuda": ([], _I),
    "ccs_ErrorString_cuda": ([_I], ctypes.c_char_p),
    "ccs_Version_cuda": ([], ctypes.c_char_p),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """Load lib/libccs_cuda.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("the CUDA library %s is not built; run `python -m halfedgecatmullclark_b200.build`"
                           % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def check(code: int, where: str) -> None:
    if code != CCS_OK:
        raise CcsError(code, where)
