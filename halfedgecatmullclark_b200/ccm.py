"""``.ccm`` cage files: reader and writer (CatmullClark.h:3085-3269).

File layout, little-endian, as the reference's x86-64 build writes it:

* a 32-byte header: int64 magic (the 8 bytes ``cc_Mesh1``, :3092-3100),
  then vertexCount, uvCount, halfedgeCount, edgeCount, faceCount as int32,
  then 4 bytes of struct padding (``ccm__Header``, :3111-3118);
* then, in this order (``ccm__ReadData``, :3162-3179): vertex->halfedge,
  edge->halfedge, face->halfedge maps (int32), vertex points (3 x f32),
  uvs (2 x f32), creases (12 B records, one per edge), halfedges (28 B).

Errors follow the reference's convention of returning nothing rather than
aborting: ``load`` raises ``CcmError`` where ``ccm_Load`` returns NULL.
"""
from __future__ import annotations

import struct

import numpy as np

from .mesh import CREASE_DTYPE, HALFEDGE_DTYPE, Cage

MAGIC = b"cc_Mesh1"
_HEADER = struct.Struct("<8s5i4x")
assert _HEADER.size == 32


class CcmError(ValueError):
    """Raised where the reference's ccm_Load would return NULL."""


def loads(data: bytes) -> Cage:
    if len(data) < _HEADER.size:
        raise CcmError("cc: fread failed")
    magic, V, U, H, E, F = _HEADER.unpack_from(data, 0)
    if magic != MAGIC:
        raise CcmError("cc: unsupported file")
    if min(V, U, H, E, F) < 0:
        raise CcmError("cc: data reading failed")
    sizes = [(V, np.int32), (E, np.int32), (F, np.int32), (3 * V, np.float32),
             (2 * U, np.float32), (E, CREASE_DTYPE), (H, HALFEDGE_DTYPE)]
    off = _HEADER.size
    out = []
    for n, dt in sizes:
        nbytes = n * np.dtype(dt).itemsize
        if off + nbytes > len(data):
            raise CcmError("cc: data reading failed")
        out.append(np.frombuffer(data, dtype=dt, count=n, offset=off).copy())
        off += nbytes
    v2h, e2h, f2h, pts, uvs, creases, halfedges = out
    return Cage(pts.reshape(-1, 3), halfedges, creases, v2h, e2h, f2h, uvs.reshape(-1, 2))


def load(path: str) -> Cage:
    """Read a ``.ccm`` file (``ccm_Load``, CatmullClark.h:3186-3220)."""
    try:
        with open(path, "rb") as fh:
            data = fh.read()
    except OSError as exc:
        raise CcmError("cc: fopen failed") from exc
    return loads(data)


def dumps(cage: Cage) -> bytes:
    parts = [_HEADER.pack(MAGIC, cage.V, cage.U, cage.H, cage.E, cage.F),
             cage.v2h.tobytes(), cage.e2h.tobytes(), cage.f2h.tobytes(),
             cage.vertex_points.astype(np.float32).tobytes(), cage.uvs.astype(np.float32).tobytes(),
             cage.creases.tobytes(), cage.halfedges.tobytes()]
    return b"".join(parts)


def save(cage: Cage, path: str) -> None:
    """Write a ``.ccm`` file (``ccm_Save``, CatmullClark.h:3227-3269)."""
    with open(path, "wb") as fh:
        fh.write(dumps(cage))


def load_pinned(path: str) -> Cage:
    """Read a ``.ccm`` file with the C library's loader (``ccs_LoadCage_cuda``).

    The returned cage's arrays are views of one page-locked host block (plain
    host memory where the CUDA runtime cannot pin), so ``Subd`` uploads them
    by DMA with no staging copy.  The block is released with the cage.
    """
    from . import _native as N
    from .mesh import cage_of_block

    L = N.lib()
    ptr = L.ccs_LoadCage_cuda(path.encode())
    if not ptr:
        code = L.ccs_LastError_cuda()
        raise CcmError("cc: cannot load %s (%s)" % (path, L.ccs_ErrorString_cuda(code).decode()))
    return cage_of_block(ptr)


def save_native(cage: Cage, path: str) -> None:
    """Write a ``.ccm`` file with the C library's writer (``ccs_SaveCage_cuda``)."""
    import ctypes

    from . import _native as N
    m = cage.as_cc_mesh()
    N.check(N.lib().ccs_SaveCage_cuda(ctypes.byref(m), path.encode()), "ccs_SaveCage_cuda")
