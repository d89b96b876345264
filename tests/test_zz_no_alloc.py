"""The allocation-free adjoint entry point, through the C ABI.

ccs_AdjointPointsDeviceNoAlloc_cuda serves callers that cannot let the
library call cudaMalloc (a CUDA graph being recorded by stream capture, an
application pool allocator that owns the device memory, a loop that forbids
allocation).  It runs the same adjoint kernels as
ccs_AdjointPointsDevice_cuda with a fixed 16 MiB array compiled into the
library as their working buffer.  These tests check, on two calls in a row,
that its gradient equals the allocating entry point's (within the float
atomics' reordering), that on a subd the allocating adjoint never touched it
leaves the device's free memory unchanged, and that a subd too large for the
array is refused.  The file is named to be collected last.
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


def test_no_alloc_adjoint_on_a_fresh_subd_allocates_nothing():
    """The property the entry point exists for.  On a subd on which the
    allocating adjoint has never run (so it has no working buffer of its own),
    the no-alloc call leaves the device's free memory unchanged, where the
    allocating entry point's first call takes cumV x 3 floats (15.6 MB here).
    Its gradient then equals the allocating adjoint's, run afterwards, on two
    calls in a row."""
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(int(stream.cuda_stream))
    # warm-up on another subd: the first call on the device looks the array up
    wa = configs.mixed_torus(nu=8, nv=8, strip=2, depth=3, seed=13)
    sa = _refined_subd(wa)
    ga = torch.ones((sa.cumV, 3), device="cuda")
    oa = torch.empty((wa.cage.V, 3), device="cuda")
    N.check(sa.L.ccs_AdjointPointsDeviceNoAlloc_cuda(sa.ptr, ga.data_ptr(), oa.data_ptr(), sp),
            "ccs_AdjointPointsDeviceNoAlloc_cuda")
    w = configs.mixed_torus(nu=32, nv=28, strip=6, depth=5, seed=12)
    s = _refined_subd(w)
    assert 3 * s.cumV <= SCRATCH_FLOATS and 12 * s.cumV > 10_000_000
    gen = torch.Generator(device="cuda").manual_seed(3)
    grads = [torch.randn((s.cumV, 3), device="cuda", generator=gen) for _ in range(2)]
    outs = [torch.full((w.cage.V, 3), float("nan"), device="cuda") for _ in range(2)]
    ref = torch.empty((w.cage.V, 3), device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for g, out in zip(grads, outs):       # two calls in a row, nothing allocated
        N.check(s.L.ccs_AdjointPointsDeviceNoAlloc_cuda(s.ptr, g.data_ptr(), out.data_ptr(), sp),
                "ccs_AdjointPointsDeviceNoAlloc_cuda")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 < (2 << 20), "device free memory fell by %d bytes" % (free0 - free1)
    for g, out in zip(grads, outs):
        N.check(s.L.ccs_AdjointPointsDevice_cuda(s.ptr, g.data_ptr(), ref.data_ptr(), sp),
                "ccs_AdjointPointsDevice_cuda")
        torch.cuda.synchronize()
        a, b = ref.cpu().numpy(), out.cpu().numpy()
        assert np.isfinite(b).all()
        assert rel_err(b, a) <= 1e-5
    s.close()
    sa.close()


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
