"""B200 (sm_100a) Catmull-Clark halfedge refinement.

A drop-in for the refinement hot path of jdupuy/HalfedgeCatmullClark's
CatmullClark.h: the C ABI in include/ccs_cuda.h (lib/libccs_cuda.so) keeps
the reference's cc_Mesh / cc_Subd layout and ccs_Create / ccs_Refine_* call
shapes; this package is its Python host side (cage building, .ccm files,
the Subd wrapper, the PyTorch autograd function and batching).
"""
from .mesh import Cage, cc_Mesh, cc_Subd  # noqa: F401

__all__ = ["Cage", "cc_Mesh", "cc_Subd"]
