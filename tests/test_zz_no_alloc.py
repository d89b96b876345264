"""The allocation-free adjoint entry point, through the C ABI.

ccs_AdjointPointsDeviceNoAlloc_cuda serves callers that cannot let the
library call cudaMalloc (a CUDA graph being recorded by stream capture, an
application pool allocator that owns the device memory, a loop that forbids
allocation).  It runs the same adjoint kernels as
ccs_AdjointPointsDevice_cuda with a fixed 16 MiB array compiled into the
library as their working buffer.  This test checks, on two calls in a row,
that its gradient equals the allocating entry point's, and that a subd too
large for the array is refused.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available, rel_err

pytestmark = pytest.mark.gpu

SCRATCH_FLOATS = 4 * 1024 * 1024


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def _refined_subd(w):
    from halfedgecatmullclark_b200.subd import Subd
    s = Subd(w.cage, w.depth)
    s.refine_halfedges()
    s.refine_creases()
    s.synchronize()
    return s


def test_no_alloc_adjoint_matches_allocating_adjoint():
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    w = configs.mixed_torus(nu=20, nv=16, strip=6, depth=4, seed=8)
    s = _refined_subd(w)
    assert 3 * s.cumV <= SCRATCH_FLOATS
    gen = torch.Generator(device="cuda").manual_seed(1)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(int(stream.cuda_stream))
    ref = torch.empty((w.cage.V, 3), device="cuda")
    grads = [torch.randn((s.cumV, 3), device="cuda", generator=gen) for _ in range(2)]
    for g in grads:                       # two calls in a row
        N.check(s.L.ccs_AdjointPointsDevice_cuda(s.ptr, g.data_ptr(), ref.data_ptr(), sp),
                "ccs_AdjointPointsDevice_cuda")
        out = torch.full((w.cage.V, 3), float("nan"), device="cuda")
        N.check(s.L.ccs_AdjointPointsDeviceNoAlloc_cuda(s.ptr, g.data_ptr(), out.data_ptr(), sp),
                "ccs_AdjointPointsDeviceNoAlloc_cuda")
        torch.cuda.synchronize()
        a, b = ref.cpu().numpy(), out.cpu().numpy()
        assert np.isfinite(b).all()
        assert rel_err(b, a) <= 1e-5
    s.close()


def test_no_alloc_adjoint_refuses_oversized_subd():
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    w = configs.mixed_torus(nu=32, nv=32, strip=8, depth=5, seed=9)
    s = _refined_subd(w)
    assert 3 * s.cumV > SCRATCH_FLOATS
    g = torch.zeros((s.cumV, 3), device="cuda")
    out = torch.zeros((w.cage.V, 3), device="cuda")
    sp = ctypes.c_void_p(int(torch.cuda.current_stream().cuda_stream))
    assert s.L.ccs_AdjointPointsDeviceNoAlloc_cuda(s.ptr, g.data_ptr(), out.data_ptr(), sp) == -8
    assert s.L.ccs_LastError_cuda() == -8
    s.close()
