"""Batched refinement of many cages of uneven size and depth.

``Batch`` wraps the ``ccs_Batch*_cuda`` entry points: every depth runs as one
persistent cooperative kernel over all cages still active at that depth, and
each operation replays one CUDA graph.  ``BatchRefinePoints`` is the
differentiable forward (points of every cage, every depth) with the batched
adjoint as its backward.  ``autotune`` picks the persistent grid size
(resident blocks per SM) by timing forward + adjoint, and caches the choice in
a JSON file keyed by GPU and batch shape.
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

from . import _native as N
from .mesh import CREASE_DTYPE, Cage


def _cuda_tensor(ptr: int, shape, typestr: str):
    import torch

    class _A:
        pass
    a = _A()
    a.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                  "version": 3, "strides": None, "stream": None}
    return torch.as_tensor(a, device="cuda")


class Batch:
    """Many cages refined together (one persistent launch per depth)."""

    def __init__(self, cages: list[Cage], depths: list[int], flags: int = 0):
        if len(cages) != len(depths) or not cages:
            raise ValueError("one depth per cage")
        self.L = N.lib()
        self.cages = list(cages)
        self.depths = [int(d) for d in depths]
        self._meshes = [c.as_cc_mesh() for c in self.cages]
        arr = (ctypes.c_void_p * len(self.cages))(*[ctypes.addressof(m) for m in self._meshes])
        dep = (ctypes.c_int32 * len(self.depths))(*self.depths)
        out = ctypes.c_void_p()
        N.check(self.L.ccs_BatchCreate_cuda(arr, dep, len(self.cages), flags, ctypes.byref(out)),
                "ccs_BatchCreate_cuda")
        self.ptr = out.value
        self.info = [self.cage_info(i) for i in range(len(self.cages))]
        self._arrays = None

    def __len__(self):
        return len(self.cages)

    def cage_info(self, i: int) -> dict:
        info = N.BatchCageInfo()
        N.check(self.L.ccs_BatchCageInfo_cuda(self.ptr, i, ctypes.byref(info)), "ccs_BatchCageInfo_cuda")
        return {k: int(getattr(info, k)) for k, _ in N.BatchCageInfo._fields_}

    # -- operations ----------------------------------------------------------
    def refine(self, mode: str = "scatter"):
        N.check(self.L.ccs_BatchRefine_cuda(self.ptr, N.POINT_MODES[mode]), "ccs_BatchRefine_cuda")

    def refine_points(self, mode: str = "scatter"):
        N.check(self.L.ccs_BatchRefinePoints_cuda(self.ptr, N.POINT_MODES[mode]), "ccs_BatchRefinePoints_cuda")

    def adjoint(self):
        N.check(self.L.ccs_BatchAdjointPoints_cuda(self.ptr), "ccs_BatchAdjointPoints_cuda")

    def adjoint_distance(self, target):
        """grad_cage_points = S^T (P - target) (ccs_BatchAdjointDistance_cuda):
        the adjoint of a fitting loss's gradient direction, with the finest
        levels' P - target formed inside the first adjoint step.  `target`: a
        float32 CUDA tensor in the points' layout, kept alive by the caller."""
        assert target.is_cuda and target.dtype.is_floating_point and target.is_contiguous()
        N.check(self.L.ccs_BatchAdjointDistance_cuda(self.ptr, target.data_ptr()),
                "ccs_BatchAdjointDistance_cuda")

    def synchronize(self):
        N.check(self.L.ccs_BatchSynchronize_cuda(self.ptr), "ccs_BatchSynchronize_cuda")

    def set_stream(self, stream) -> None:
        handle = getattr(stream, "cuda_stream", stream)
        N.check(self.L.ccs_BatchSetStream_cuda(self.ptr, ctypes.c_void_p(int(handle) if handle else 0)),
                "ccs_BatchSetStream_cuda")

    def set_schedule(self, blocks_per_sm: int, split: bool | None = None) -> None:
        N.check(self.L.ccs_BatchSetSchedule_cuda(self.ptr, int(blocks_per_sm)), "ccs_BatchSetSchedule_cuda")
        if split is not None:
            N.check(self.L.ccs_BatchSetLaunchMode_cuda(self.ptr, 1 if split else 0), "ccs_BatchSetLaunchMode_cuda")

    # -- device buffers as torch tensors (no copy) ----------------------------
    def arrays(self) -> dict:
        if self._arrays is None:
            a = N.BatchArrays()
            N.check(self.L.ccs_BatchGetArrays_cuda(self.ptr, ctypes.byref(a)), "ccs_BatchGetArrays_cuda")
            self._arrays = {
                "halfedges": _cuda_tensor(a.halfedges, (a.halfedgeCount, 4), "<i4"),
                "creases": _cuda_tensor(a.creases, (a.creaseCount, 3), "<i4"),
                "points": _cuda_tensor(a.points, (a.pointCount, 3), "<f4"),
                "cage_points": _cuda_tensor(a.cagePoints, (a.cagePointCount, 3), "<f4"),
                "grad_points": _cuda_tensor(a.gradPoints, (a.pointCount, 3), "<f4"),
                "grad_cage_points": _cuda_tensor(a.gradCagePoints, (a.cagePointCount, 3), "<f4"),
            }
        return self._arrays

    def cage_slice(self, i: int) -> slice:
        inf = self.info[i]
        return slice(inf["cagePointOffset"], inf["cagePointOffset"] + inf["cagePointCount"])

    def point_slice(self, i: int, finest: bool = False) -> slice:
        inf = self.info[i]
        if finest:
            return slice(inf["finestPointOffset"], inf["finestPointOffset"] + inf["finestPointCount"])
        return slice(inf["pointOffset"], inf["pointOffset"] + inf["pointCount"])

    def download(self, i: int):
        """(halfedges, creases, points) of cage i as numpy arrays."""
        arr = self.arrays()
        inf = self.info[i]
        he = arr["halfedges"][inf["halfedgeOffset"]: inf["halfedgeOffset"] + inf["halfedgeCount"]]
        cr = arr["creases"][inf["creaseOffset"]: inf["creaseOffset"] + inf["creaseCount"]]
        pts = arr["points"][self.point_slice(i)]
        self.synchronize()
        return (he.cpu().numpy(), np.ascontiguousarray(cr.cpu().numpy()).view(CREASE_DTYPE).reshape(-1),
                pts.cpu().numpy())

    def close(self):
        if getattr(self, "ptr", None):
            self._arrays = None
            self.L.ccs_BatchRelease_cuda(self.ptr)
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


def _make_function():
    import torch

    class BatchRefinePoints(torch.autograd.Function):
        """All cages' cage points (concatenated) -> all cages' refined points."""

        @staticmethod
        def forward(ctx, cage_points, batch: Batch):
            arr = batch.arrays()
            batch.set_stream(torch.cuda.current_stream())
            arr["cage_points"].copy_(cage_points.detach().to(torch.float32))
            batch.refine_points()
            ctx.batch = batch
            return arr["points"].clone()

        @staticmethod
        def backward(ctx, grad):
            batch = ctx.batch
            arr = batch.arrays()
            batch.set_stream(torch.cuda.current_stream())
            arr["grad_points"].copy_(grad.to(torch.float32))
            batch.adjoint()
            return arr["grad_cage_points"].clone(), None

    return BatchRefinePoints


_FN = None


def refine_points(cage_points, batch: Batch):
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN.apply(cage_points, batch)


# ---------------------------------------------------------------------------
# autotuner
# ---------------------------------------------------------------------------
def cache_path() -> str:
    return os.environ.get("CCS_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "halfedgecatmullclark_b200",
                                       "autotune.json"))


def _key(batch: Batch) -> str:
    import torch
    name = torch.cuda.get_device_name()
    sh = sum(inf["halfedgeCount"] for inf in batch.info)
    return "%s|cages=%d|halfedges=%d|maxdepth=%d" % (name, len(batch), sh, max(batch.depths))


def time_fwd_adj(batch: Batch, iters: int = 5, stream=None) -> float:
    """Mean ms of one forward (points) + adjoint, CUDA events on `stream`
    (default: the current torch stream), which the batch is bound to."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    batch.set_stream(s)
    batch.refine_points()
    batch.adjoint()
    batch.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(iters):
        batch.refine_points()
        batch.adjoint()
    b.record(s)
    batch.synchronize()
    return a.elapsed_time(b) / iters


def autotune(batch: Batch, candidates=(0, 2, 4, 6, 8), iters: int = 5, use_cache: bool = True,
             stream=None, modes=(False, True)) -> dict:
    """Choose the launch schedule -- one cooperative launch per depth or one
    launch per section (`modes`: split or not) -- and the resident blocks
    per SM of the persistent kernels, by timing forward + adjoint on `stream`
    (default the current torch stream; the batch stays bound to it)."""
    path = cache_path()
    key = _key(batch)
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            with open(path) as fh:
                cache = json.load(fh)
        except Exception:
            cache = {}
    if use_cache and key in cache:
        batch.set_schedule(cache[key]["blocks_per_sm"], bool(cache[key].get("split", False)))
        return dict(cache[key], cached=True)
    results = {}
    for split in modes:
        for c in candidates:
            batch.set_schedule(c, split)
            results[(split, c)] = time_fwd_adj(batch, iters, stream)
    best = min(results, key=results.get)
    batch.set_schedule(best[1], best[0])
    entry = {"blocks_per_sm": best[1], "split": best[0], "ms": results[best],
             "tried": {("split/%d" if k[0] else "fused/%d") % k[1]: v for k, v in results.items()}}
    cache[key] = entry
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(cache, fh, indent=1)
    except OSError:
        pass
    return dict(entry, cached=False)
