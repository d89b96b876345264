"""FP32 accuracy of the CUDA points against the FP64 oracle of the same rule.

For config 1 (the quad torus, depth 4) and the headline mixed-crease torus at
depth 6, the test states the max-norm relative error (max |p - p64| / max |p64|)
and the RMS error relative to the same scale for three FP32 results:

* the default path (float atomics in the GPU's order);
* the deterministic path (the reference's one-thread summation order);
* the oracle in FP32, i.e. the reference's own order of operations.

It prints one line per result (run with ``-s`` to see them) and asserts the
bar: the default path is within 1e-5 and no less accurate than the
reference's FP32 order by more than a small factor, the deterministic path
equals the FP32 oracle bit for bit, and, where the reference is built, the
default path is within 1e-5 of the reference's own multi-threaded
ccs_Refine_Scatter on the same cage and depth.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

TOL_POINTS = 1e-5


@pytest.fixture(scope="module", autouse=True)
def built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build
    build.build()


def _errors(p, p64):
    d = p.astype(np.float64) - p64
    scale = float(np.abs(p64).max())
    return float(np.abs(d).max()) / scale, float(np.sqrt(np.mean(d * d))) / scale


def _gpu_points(cage, depth, flags):
    from halfedgecatmullclark_b200.subd import Subd
    with Subd(cage, depth, flags) as s:
        s.refine_scatter()
        s.download()
        return s.halfedges().copy(), s.creases().copy(), s.points().copy()


@pytest.mark.slow
@pytest.mark.parametrize("config", ["torus_quads_d4", "mixed_torus_d6"])
def test_error_report_against_fp64(config):
    from halfedgecatmullclark_b200 import _native as N, configs
    from oracle import oracle
    w = configs.torus_quads() if config == "torus_quads_d4" else configs.mixed_torus()
    he, cr, p_def = _gpu_points(w.cage, w.depth, 0)
    _, _, p_det = _gpu_points(w.cage, w.depth, N.FLAG_DETERMINISTIC)
    # the topology was checked bit-exact against the oracle elsewhere; the
    # oracle's point rules run on it in both precisions
    p64 = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float64)
    o32 = oracle.refine_points(w.cage, w.depth, he, cr, "scatter", np.float32)
    rows = {"default": _errors(p_def, p64), "deterministic": _errors(p_det, p64),
            "fp32 reference order": _errors(o32, p64)}
    for name, (mx, rms) in rows.items():
        print("fp64 error %s %s (%d points): max %.3e rms %.3e" % (config, name, p64.shape[0], mx, rms))
    assert rows["default"][0] <= TOL_POINTS
    assert rows["default"][0] <= 4 * rows["fp32 reference order"][0] + 1e-7
    assert np.array_equal(p_det.view(np.uint32), o32.view(np.uint32))
    # against the reference's own multi-threaded ccs_Refine_Scatter, when built
    from oracle import refimpl
    if refimpl.available():
        refimpl.set_threads(refimpl.max_threads())
        s = refimpl.RefSubd(w.cage, w.depth)
        try:
            s.refine("scatter")
            ref = s.points().copy()
            assert np.array_equal(s.halfedges()[:, :3], he[:, :3])
        finally:
            s.close()
        d = p_def.astype(np.float64) - ref.astype(np.float64)
        scale = float(np.abs(ref).max())
        mx, rms = float(np.abs(d).max()) / scale, float(np.sqrt(np.mean(d * d))) / scale
        print("fp32 reference %s default vs ccs_Refine_Scatter (%d threads): max %.3e rms %.3e"
              % (config, refimpl.max_threads(), mx, rms))
        assert mx <= TOL_POINTS
