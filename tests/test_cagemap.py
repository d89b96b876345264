"""The cage step as a sparse linear map (ccs_CageStepMatrix_cuda, host
only): the map the default pass evaluates as its cage step equals the FP64
oracle's cage rules (CatmullClark.h:1437-1991, creased and NoCreases scatter)
on every cage the tests use, and its transpose equals the oracle's adjoint
of the cage level."""
import numpy as np
import pytest

from conftest import ccm_paths, rel_err, small_cages


def _cages(small_workloads):
    from halfedgecatmullclark_b200 import ccm, configs
    out = [(w.name, w.cage) for w in small_workloads]
    out += small_cages()
    out.append(("mixed_torus_64x64", configs.mixed_torus(depth=1).cage))
    out += [(p.rsplit("/", 1)[-1], ccm.load(p)) for p in ccm_paths()]
    return out


def _apply(rp, col, w, x):
    rows = len(rp) - 1
    out = np.zeros((rows, x.shape[1]))
    r = np.repeat(np.arange(rows), np.diff(rp))
    np.add.at(out, r, w.astype(np.float64)[:, None] * x[col])
    return out


@pytest.mark.parametrize("mode", ["scatter", "nocreases_scatter"])
def test_cage_step_matrix_matches_oracle(small_workloads, mode):
    from halfedgecatmullclark_b200.subd import cage_step_matrix
    from oracle import oracle
    for name, cage in _cages(small_workloads):
        rp, col, w = cage_step_matrix(cage, mode)
        assert len(rp) - 1 == cage.V + cage.F + cage.E and np.all(np.diff(rp) > 0)
        p1 = _apply(rp, col, w, cage.vertex_points.astype(np.float64))
        he, cr = oracle.refine_topology(cage, 1)
        ref = oracle.refine_points(cage, 1, he, cr, mode, np.float64)
        assert rel_err(p1, ref) <= 1e-6, (name, mode, rel_err(p1, ref))


def test_cage_step_transpose_is_the_adjoint(small_workloads):
    from halfedgecatmullclark_b200.subd import cage_step_matrix
    from oracle import oracle
    rng = np.random.default_rng(2)
    for name, cage in _cages(small_workloads):
        rp, col, w = cage_step_matrix(cage, "scatter", transpose=True)
        assert len(rp) - 1 == cage.V
        he, cr = oracle.refine_topology(cage, 1)
        g = rng.normal(size=(cage.V + cage.F + cage.E, 3))
        got = _apply(rp, col, w, g)
        ref = oracle.adjoint(cage, 1, he, cr, g)
        assert rel_err(got, ref) <= 1e-6, (name, rel_err(got, ref))
