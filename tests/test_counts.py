"""Count / stride algebra (CatmullClark.h:465-585, :815-936).

Known answers: the per-depth and cumulative counts the reference computes
for its sample cages (recorded in tests/golden/reference_digests.json), the
self-check of examples/mesh_info.c:365-392 (cumulative count == sum of the
per-depth counts), and the int32 ceiling of the cc_Subd layout.  The C ABI's
ccs_LevelCounts_cuda is host arithmetic and runs without a GPU.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, ccm_paths


def test_oracle_counts_match_reference_known_answers():
    from halfedgecatmullclark_b200 import ccm
    from oracle import oracle
    with open(os.path.join(ROOT, "tests", "golden", "reference_digests.json")) as fh:
        g = json.load(fh)["ccm"]
    paths = ccm_paths()
    if not paths:
        pytest.skip("sample cages not available")
    for p in paths:
        ref = g[os.path.basename(p)]["counts"]
        cnt = oracle.counts(ccm.load(p), 5)
        for k in ("H", "F", "E", "V", "C", "cumH", "cumF", "cumE", "cumV", "cumC"):
            assert cnt[k] == ref[k], (p, k)


def test_cumulative_is_sum_of_levels(small_workloads):
    from oracle import oracle
    for w in small_workloads:
        cnt = oracle.counts(w.cage, 5)
        for d in range(6):
            for k, c in (("H", "cumH"), ("V", "cumV"), ("C", "cumC"), ("E", "cumE"), ("F", "cumF")):
                assert cnt[c][d] == sum(cnt[k][1:d + 1]), (w.name, k, d)


def test_capi_counts_match_oracle(small_workloads):
    from halfedgecatmullclark_b200.subd import level_counts
    from oracle import oracle
    for w in small_workloads:
        D = 5
        lc = level_counts(w.cage, D)
        cnt = oracle.counts(w.cage, D)
        for d in range(D + 1):
            for k in "HFEVC":
                assert lc[d][k] == cnt[k][d]
            if d:
                assert lc[d]["cumH"] == cnt["cumH"][d - 1]
                assert lc[d]["cumV"] == cnt["cumV"][d - 1]
                assert lc[d]["cumC"] == cnt["cumC"][d - 1]


def test_overflow_is_refused():
    """Depth 6 of the 256x256 grid needs 4.7e9 halfedges: beyond int32."""
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200.subd import level_counts, max_supported_depth
    w = configs.height_grid(n=256, depth=5)
    assert max_supported_depth(w.cage) == 5
    level_counts(w.cage, 5)
    with pytest.raises(N.CcsError) as ei:
        level_counts(w.cage, 6)
    assert ei.value.code == -3


def test_paper_formulas_small_cage():
    """F^{d+1} = H^d, E^{d+1} = 2E^d + H^d, V^{d+1} = V^d + E^d + F^d."""
    from halfedgecatmullclark_b200 import configs
    from oracle import oracle
    w = configs.mixed_torus(nu=8, nv=8, strip=3, depth=5)
    c = oracle.counts(w.cage, 6)
    for d in range(6):
        assert c["F"][d + 1] == c["H"][d]
        assert c["E"][d + 1] == 2 * c["E"][d] + c["H"][d]
        assert c["V"][d + 1] == c["V"][d] + c["E"][d] + c["F"][d]
        assert c["H"][d + 1] == 4 * c["H"][d]
        assert c["C"][d + 1] == 2 * c["C"][d]
    assert np.all(np.diff(c["cumH"]) > 0)
