"""Cage building and .ccm files against the reference's own code."""
import numpy as np
import pytest

from conftest import ccm_paths

FIELDS = [("points", "vertex_points"), ("uvs", "uvs"), ("halfedges", "halfedges"), ("creases", "creases"),
          ("v2h", "v2h"), ("e2h", "e2h"), ("f2h", "f2h")]


def same(cage, ref):
    return {k: np.array_equal(getattr(cage, a).view(np.uint8), ref[k].view(np.uint8)) for k, a in FIELDS}


def test_builder_matches_reference_obj_loader():
    """build_cage == examples/obj_to_ccm.c LoadObj on the same OBJ text."""
    from oracle import refimpl
    if not refimpl.available():
        pytest.skip("reference not built")
    from halfedgecatmullclark_b200 import configs
    ws = [configs.torus_quads(), configs.mixed_torus(), configs.fitting_cage(),
          configs.mixed_torus(nu=7, nv=5, strip=3, seed=9), configs.height_grid(n=20, seed=2)]
    ws += configs.batch_cages(count=3, fmax=300, seed=4)
    for w in ws:
        ref = refimpl.load_obj_text(w.obj())
        ok = same(w.cage, ref)
        assert all(ok.values()), (w.name, ok)


def test_ccm_roundtrip_and_reference_loader(tmp_path):
    from halfedgecatmullclark_b200 import ccm
    from oracle import refimpl
    paths = ccm_paths()
    if not paths:
        pytest.skip("sample cages not available")
    for p in paths:
        data = open(p, "rb").read()
        cage = ccm.loads(data)
        again = ccm.dumps(cage)
        # bytes 28..31 are the header's struct padding, which ccm_Save writes
        # uninitialised (CatmullClark.h:3111-3118, :3244)
        assert again[:28] == data[:28] and again[32:] == data[32:]
        out = str(tmp_path / "x.ccm")
        ccm.save(cage, out)
        if refimpl.available():
            ref = refimpl.load_ccm(out)
            assert all(same(cage, ref).values())


def test_ccm_errors(tmp_path):
    from halfedgecatmullclark_b200 import ccm, configs
    w = configs.torus_quads()
    data = ccm.dumps(w.cage)
    with pytest.raises(ccm.CcmError):
        ccm.loads(b"xx")
    with pytest.raises(ccm.CcmError):
        ccm.loads(b"cc_MeshX" + data[8:])
    with pytest.raises(ccm.CcmError):
        ccm.loads(data[:-5])
    with pytest.raises(ccm.CcmError):
        ccm.load(str(tmp_path / "missing.ccm"))
    assert ccm.dumps(ccm.loads(data)) == data


def test_builder_rejects_bad_input():
    from halfedgecatmullclark_b200.cage import build_cage
    pts = np.zeros((4, 3), np.float32)
    with pytest.raises(ValueError):
        build_cage(pts, [[0, 1]])                       # degenerate face
    with pytest.raises(ValueError):
        build_cage(pts, [[0, 1, 2], [0, 1, 3]])          # directed edge 0->1 twice
    with pytest.raises(ValueError):
        build_cage(pts, [[0, 1, 7]])                     # vertex out of range


def test_builder_conventions_on_a_single_quad():
    """One open quad: every edge is a boundary (sharpness 16), twins -1."""
    from halfedgecatmullclark_b200.cage import build_cage
    pts = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    c = build_cage(pts, [[0, 1, 2, 3]])
    assert c.H == 4 and c.E == 4 and c.F == 1
    assert np.all(c.halfedges["twinID"] == -1)
    assert np.all(c.creases["sharpness"] == 16.0)
    assert list(c.halfedges["nextID"]) == [1, 2, 3, 0]
    assert list(c.halfedges["prevID"]) == [3, 0, 1, 2]
    assert list(c.e2h) == [0, 1, 2, 3]
    # crease links are made only through closed vertex rings
    # (examples/obj_to_ccm.c:219-249), so boundary creases stay self-linked
    assert list(c.creases["nextID"]) == [0, 1, 2, 3]
    assert list(c.creases["prevID"]) == [0, 1, 2, 3]


def test_native_ccm_loader_and_writer(tmp_path):
    """ccs_LoadCage_cuda / ccs_SaveCage_cuda against the Python reader and
    the files' own bytes (header padding aside)."""
    from halfedgecatmullclark_b200 import build, ccm
    build.build()
    paths = ccm_paths()
    if not paths:
        pytest.skip("sample cages not available")
    for p in paths:
        ref = ccm.load(p)
        cage = ccm.load_pinned(p)
        for _, a in FIELDS:
            assert np.array_equal(getattr(cage, a).view(np.uint8), getattr(ref, a).view(np.uint8)), (p, a)
        out = str(tmp_path / "native.ccm")
        ccm.save_native(cage, out)
        data, again = open(p, "rb").read(), open(out, "rb").read()
        assert again[:28] == data[:28] and again[28:32] == b"\0" * 4 and again[32:] == data[32:]
        del cage


def test_native_ccm_loader_errors(tmp_path):
    from halfedgecatmullclark_b200 import _native as N, build, ccm, configs
    build.build()
    data = ccm.dumps(configs.torus_quads().cage)
    bad = {"magic": b"cc_MeshX" + data[8:], "short": data[:-5], "tiny": b"xx",
           "negative": data[:8] + (-1).to_bytes(4, "little", signed=True) + data[12:]}
    for name, blob in bad.items():
        path = tmp_path / (name + ".ccm")
        path.write_bytes(blob)
        with pytest.raises(ccm.CcmError):
            ccm.load_pinned(str(path))
        assert N.lib().ccs_LastError_cuda() == -1          # CCS_ERR_ARG
    with pytest.raises(ccm.CcmError):
        ccm.load_pinned(str(tmp_path / "missing.ccm"))
    good = tmp_path / "good.ccm"
    good.write_bytes(data)
    assert ccm.dumps(ccm.load_pinned(str(good))) == data
    N.lib().ccs_ReleaseCage_cuda(None)                    # NULL is a no-op


@pytest.mark.gpu
def test_subd_from_pinned_cage_matches():
    """A subd made from a ccs_LoadCage_cuda cage (DMA upload from the file's
    page-locked block) refines exactly like one from the Python reader."""
    from conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    from halfedgecatmullclark_b200 import build, ccm
    from halfedgecatmullclark_b200.subd import Subd
    build.build()
    paths = ccm_paths()
    if not paths:
        pytest.skip("sample cages not available")
    for p in paths[:4]:
        res = []
        for cage in (ccm.load(p), ccm.load_pinned(p)):
            with Subd(cage, 2, 4) as s:                  # deterministic: bit-comparable
                s.refine("scatter")
                s.download()
                res.append((s.halfedges(), s.creases(), s.points()))
        for a, b in zip(*res):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), p
