"""Algorithmic byte counts of the refinement kernels (the roofline numerators).

Every figure counts each unique input read once and each output written
once, in the packed layout (16-byte halfedge records, or 12 with
CCS_FLAG_NO_UV; 12-byte creases; 12-byte points).  ``level_bytes`` is the
minimum for a whole refinement step d -> d+1 (the per-depth GB/s figure):
when the step's point pass is fused with its topology (one launch that
reads each record once: the default pass at depth >= 2) the records are
counted once; when the point pass runs as a launch of its own it reads them
again, and ``fused=False`` adds that second read.  ``kernel_bytes`` is the
per-launch figure of one kernel, which defines its achieved bandwidth.
"""
from __future__ import annotations


def level_bytes(lv: dict, nxt: dict, rec: int = 16, uv: bool = True, cage: bool = False,
                cage_uvs: int = 0, topology: bool = True, fused: bool = False) -> int:
    """Minimum HBM bytes of one full refinement step (topology, creases, points);
    with topology=False, of its points alone on a refined topology.  With
    fused=True the point pass shares the topology's single read of the
    records."""
    H, V, C = lv["H"], lv["V"], lv["C"]
    Vn = nxt["V"]
    if not topology:
        return int(12 * V + 12 * Vn + 4 * C + (28 if cage else rec) * H)
    if cage:
        topo = 28 * H + 4 * rec * H + 8 * cage_uvs
    else:
        topo = rec * H + 4 * rec * H
    creases = 12 * C + 24 * C
    points = 12 * V + 12 * Vn + 4 * C + (0 if fused else (28 if cage else rec) * H)
    return int(topo + creases + points)


def kernel_bytes(kernel: str, lv: dict, rec: int = 16, prev: dict | None = None, units: int | None = None) -> int:
    """Per-launch algorithmic bytes of one kernel at parent depth `lv`
    (`prev` = the level before it, which gives the exact count of older
    vertices at depth 1, where the quad-structure count below does not
    hold; `units` = the launch's own item count where it is not a level's:
    the statistics entries of every level for "cage_side" and the
    every-level "ring_stats" launch; the older vertices of the ring walks for
    "exact_points" and "old_vertices")."""
    H, V, F, E, C = lv["H"], lv["V"], lv["F"], lv["E"], lv["C"]
    if kernel == "cage_side":
        # cage records in, 4 child records out, cage creases in and their
        # children out, one float4 of shape statistics per entry out
        return int(28 * H + 4 * rec * H + 36 * C + 16 * (units or 0))
    if kernel in ("topology", "uvs"):
        return int(rec * H + 4 * rec * H)
    if kernel == "creases":
        return int(36 * C)
    if kernel == "face_points":
        return int(rec * H + 12 * V + 12 * F)
    if kernel == "edge_points":
        return int(rec * H + 12 * V + 12 * F + 12 * C + 12 * E)
    if kernel == "vertex_points":
        return int(rec * H + 12 * V + 12 * F + 12 * E + 12 * C + 12 * V)
    if kernel == "clear":
        return int(12 * V)
    if kernel == "level_fused":
        # records in + children out + creases in and out + points in + face
        # and edge points out + the cleared vertex slots
        return int(rec * H + 4 * rec * H + 36 * C + 12 * V + 12 * F + 12 * E + 12 * V)
    # depth d >= 2: F(d-1) = H / 16 face centres and E(d-1) = (E - H / 4) / 2
    # edge midpoints; the rest of the V vertices are older
    nb = H // 16 + (E - H // 4) // 2
    if kernel == "level_points":
        # records + crease records + face and edge points + points in, the
        # older vertices' ring statistics (16 B), vertex points out
        return int(rec * H + 12 * C + 12 * F + 12 * E + 12 * V + 16 * max(V - nb, 0) + 12 * V)
    if kernel in ("level_step", "level_step_points"):
        # one launch for the whole default step: records in (+ children out
        # and the creases with the topology), points in, face, edge and
        # vertex points out, the older vertices' ring statistics and the
        # level's crease records; the slots cleared for the next level are
        # not counted (none at the last level)
        topo = 4 * rec * H + 36 * C if kernel == "level_step" else 12 * C
        return int(rec * H + topo + 12 * V + 12 * F + 12 * E + 12 * V + 16 * max(V - nb, 0))
    if kernel == "adj_step":
        # one adjoint pass of a step: records, the gradients of depth d+1
        # (vertex, face and edge slots), the older vertices' statistics and
        # the crease records in; the gradients of depth d out
        return int(rec * H + 12 * (V + F + E) + 16 * max(V - nb, 0) + 12 * C + 12 * V)
    if kernel == "ring_stats":
        # shape half (k_shape_stats): valence and boundary from the vertex
        # numbering and the cage alone -- no level data read; one float4 per
        # older vertex out (every level's entries when `units` is given).
        if units is not None:
            return int(16 * units)
        return int(16 * (prev["V"] if prev is not None else max(V - nb, 0)))
    if kernel == "crease_stats":
        # crease half (k_crease_stats): the level's crease records in; the
        # atomics of its creased edges go to the statistics already written
        return int(12 * C)
    # the exact pass: `units` = the older vertices the ring walks take (all
    # V - nb, or from depth 3 only those of depth d-2, the per-face pass
    # summing the centres and edge midpoints of depth d-2 as well)
    older = max(V - nb, 0) if units is None else int(units)
    if kernel == "exact_points":
        # records + crease records + face and edge points in; the points of
        # its vertices in and out
        return int(rec * H + 12 * C + 12 * F + 12 * E + 24 * (V - older))
    if kernel == "old_vertices":
        # records of children 0 and 3 (the ring walk), the ring's face and
        # edge points (one member per halfedge of the walks' depth: H / 4,
        # or H / 16 from depth d-2), the points in and out
        members = H // 4 if older >= V - nb else H // 16
        return int(2 * rec * members + 24 * members + 24 * older)
    if kernel == "adjoint":
        return int(rec * H + 12 * C + 12 * (V + F + E) + 12 * V)
    return 0


def total_halfedges(levels: list[dict]) -> int:
    """Refined halfedges of depths 1..D (the unit of the headline metric)."""
    return int(sum(lv["H"] for lv in levels[1:]))
