"""PyTorch extension: differentiable refinement of cage points.

For a fixed topology and fixed crease sharpness, the refined points of every
level are linear in the cage points (each branch of the vertex rule depends
only on topology and sharpness).  ``RefinePoints`` runs the forward scatter
rule with the CUDA kernels (``ccs_RefinePointsDevice_cuda``) and its
backward with the hand-written adjoint kernels
(``ccs_AdjointPointsDevice_cuda``: the transposed rules run as gathers over
the refined halfedges, deepest level first).  The forward saves no tensor:
the adjoint needs only the subd's level offsets and its device topology.

Both run on the caller's current CUDA stream, so the function composes with
torch streams.
"""
from __future__ import annotations

import torch

from . import _native as N
from .subd import Subd


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


class RefinePoints(torch.autograd.Function):
    """cage points (V0 x 3, float32, cuda) -> packed points of depths 1..D."""

    @staticmethod
    def forward(ctx, cage_points: torch.Tensor, subd: Subd, mode: int = N.POINTS_SCATTER):
        if not cage_points.is_cuda or cage_points.dtype != torch.float32:
            raise TypeError("cage points must be a float32 CUDA tensor")
        x = cage_points.contiguous()
        if x.shape != (subd.cage.V, 3):
            raise ValueError("expected cage points of shape (%d, 3)" % subd.cage.V)
        out = torch.empty((subd.cumV, 3), dtype=torch.float32, device=x.device)
        N.check(subd.L.ccs_RefinePointsDevice_cuda(subd.ptr, x.data_ptr(), out.data_ptr(), mode, _stream()),
                "ccs_RefinePointsDevice_cuda")
        ctx.subd = subd
        ctx.mode = mode
        return out

    @staticmethod
    def backward(ctx, grad):
        subd = ctx.subd
        if ctx.mode != N.POINTS_SCATTER:
            raise NotImplementedError("the adjoint covers the creased scatter rule")
        g = grad.contiguous().to(torch.float32)
        gc = torch.empty((subd.cage.V, 3), dtype=torch.float32, device=g.device)
        N.check(subd.L.ccs_AdjointPointsDevice_cuda(subd.ptr, g.data_ptr(), gc.data_ptr(), _stream()),
                "ccs_AdjointPointsDevice_cuda")
        return gc, None, None


def refine_points(cage_points: torch.Tensor, subd: Subd) -> torch.Tensor:
    """Differentiable packed points (subd.cumV x 3) of depths 1..subd.depth."""
    return RefinePoints.apply(cage_points, subd)


def level(points: torch.Tensor, subd: Subd, depth: int | None = None) -> torch.Tensor:
    """View of one depth's points inside the packed array (default: finest)."""
    return points[subd.level_slice(subd.depth if depth is None else depth, "V")]


class SubdivisionSurface(torch.nn.Module):
    """A refinement operator bound to one cage topology.

    The topology (halfedges, creases) is refined once at construction; each
    call maps cage points to the points of the finest level (or of all
    levels with ``all_levels=True``).
    """

    def __init__(self, cage, depth: int, flags: int = 0):
        super().__init__()
        self.subd = Subd(cage, depth, flags)
        self.subd.set_stream(torch.cuda.current_stream())
        self.subd.refine_halfedges()
        self.subd.refine_creases()
        self.subd.synchronize()

    def forward(self, cage_points: torch.Tensor, all_levels: bool = False) -> torch.Tensor:
        pts = refine_points(cage_points, self.subd)
        return pts if all_levels else level(pts, self.subd)
