"""Drop-in replacement of the boundary self-intersection check of the
reference's ``engine/charts.py`` (boundary_intersections, :547-608).

``boundary_intersections(U, T, max_report=1000)`` keeps the reference's
signature and result: the number of crossing pairs of the chart's directed
boundary segments, counted once per cell of the reference's uniform grid
the pair shares (cell = max(4 median segment length, extent / 512, 1e-30)),
capped at max(max_report, 1); 0 below 3 boundary segments; ValueError for
non-finite UVs (the reference fails converting the grid size to int). The
pair tests run on the GPU (uva_boundary_hits, exact FP64 without fused
multiply-add). UVs are taken as FP64: a float32 U is widened first, where
the reference would evaluate its predicate in float32.

``boundary_intersections_batch(charts, max_report=1000)`` is an addition:
one launch for a list of (U, T) charts, one count per chart (-1 where the
reference would raise).
"""
from __future__ import annotations

import numpy as np

from .. import segments


def _chart_segments(U, T):
    U = np.asarray(U, np.float64).reshape(-1, 2)
    a, b, _ = segments.directed_boundary(T)
    if len(a) and (a.min() < 0 or max(a.max(), b.max()) >= len(U)):
        raise IndexError("boundary_intersections: T names a vertex outside U")
    return U, np.stack([a, b], 1)


def boundary_intersections(U, T, max_report=1000):
    """Exact count of self-intersections of the chart's UV boundary
    (engine/charts.py:596-608)."""
    U, seg = _chart_segments(U, T)
    if len(seg) < 3:
        return 0
    out = segments.boundary_hits(U, [0, len(seg)], seg, segments.COUNT, max_report, vofs=[0, len(U)])
    if out[0] == -1:
        raise ValueError("boundary_intersections: non-finite UVs")
    return int(out[0])


def boundary_intersections_batch(charts, max_report=1000):
    """boundary_intersections of every (U, T) chart in one launch -> int64
    array (-1 for a chart with >= 3 boundary segments and non-finite UVs)."""
    Us, segs, vofs, sofs = [], [], [0], [0]
    for U, T in charts:
        Uc, seg = _chart_segments(U, T)
        Us.append(Uc)
        segs.append(seg + vofs[-1])
        vofs.append(vofs[-1] + len(Uc))
        sofs.append(sofs[-1] + len(seg))
    if not Us:
        return np.zeros(0, np.int64)
    U = np.concatenate(Us) if vofs[-1] else np.zeros((0, 2))
    seg = np.concatenate(segs) if sofs[-1] else np.zeros((0, 2), np.int64)
    return segments.boundary_hits(U, sofs, seg, segments.COUNT, max_report, vofs=vofs)
