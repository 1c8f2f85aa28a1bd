"""Oracle for the boundary self-intersection checks (test infrastructure only).

CPU restatement of engine/charts.py:547-608 (boundary_intersections,
_seg_intersections) and engine/hier.py:158-353 (boundary_directed,
charts_collide, _hit, chart_checks) of the reference. Two forms of the
segment count:

* ``seg_intersections_cells``: the reference's own procedure, pure Python
  loops (small cases): bin every segment into the cells of its box, test
  every pair inside every cell, stop at max_report.
* ``seg_intersections_pairs``: numpy over all pairs: a crossing pair adds the
  number of cells both boxes share (what the cell loop counts), capped.

Both evaluate the predicate with numpy / Python FP64 arithmetic in the
reference's operation order (no fused multiply-add). The tests pin both
against golden_segments.npz, made by running the reference itself.
"""
from __future__ import annotations

import numpy as np


def boundary_edges_oriented(T):
    """engine/param.py:59-68: directed half-edges whose reverse is absent."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]])
    b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
    if len(a) == 0:
        return a, b
    n = int(max(a.max(), b.max())) + 1
    twin = np.isin(b * n + a, a * n + b)
    return a[~twin], b[~twin]


def cross(ai, bi, aj, bj):
    """engine/charts.py:579-591 for one pair of segments (Python floats)."""
    if (ai[0] == aj[0] and ai[1] == aj[1]) or (ai[0] == bj[0] and ai[1] == bj[1]) or \
       (bi[0] == aj[0] and bi[1] == aj[1]) or (bi[0] == bj[0] and bi[1] == bj[1]):
        return False
    d1x = bi[0] - ai[0]; d1y = bi[1] - ai[1]
    d2x = bj[0] - aj[0]; d2y = bj[1] - aj[1]
    o1 = d1x * (aj[1] - ai[1]) - d1y * (aj[0] - ai[0])
    o2 = d1x * (bj[1] - ai[1]) - d1y * (bj[0] - ai[0])
    o3 = d2x * (ai[1] - aj[1]) - d2y * (ai[0] - aj[0])
    o4 = d2x * (bi[1] - aj[1]) - d2y * (bi[0] - aj[0])
    tol1 = 1e-9 * (d1x * d1x + d1y * d1y)
    tol2 = 1e-9 * (d2x * d2x + d2y * d2y)
    return ((o1 > tol1 and o2 < -tol1) or (o1 < -tol1 and o2 > tol1)) and \
           ((o3 > tol2 and o4 < -tol2) or (o3 < -tol2 and o4 > tol2))


def cross_matrix(A, B):
    """cross() for every pair (i, j) as an (m, m) bool array (numpy)."""
    with np.errstate(over="ignore", invalid="ignore"):   # huge UVs overflow like the reference's
        return _cross_matrix(np.asarray(A, np.float64), np.asarray(B, np.float64))


def _cross_matrix(A, B):
    ax, ay, bx, by = A[:, 0][:, None], A[:, 1][:, None], B[:, 0][:, None], B[:, 1][:, None]
    cx, cy, dx, dy = A[:, 0][None], A[:, 1][None], B[:, 0][None], B[:, 1][None]
    same = ((ax == cx) & (ay == cy)) | ((ax == dx) & (ay == dy)) | ((bx == cx) & (by == cy)) | ((bx == dx) & (by == dy))
    d1x = bx - ax; d1y = by - ay
    d2x = dx - cx; d2y = dy - cy
    o1 = d1x * (cy - ay) - d1y * (cx - ax)
    o2 = d1x * (dy - ay) - d1y * (dx - ax)
    o3 = d2x * (ay - cy) - d2y * (ax - cx)
    o4 = d2x * (by - cy) - d2y * (bx - cx)
    tol1 = 1e-9 * (d1x * d1x + d1y * d1y)
    tol2 = 1e-9 * (d2x * d2x + d2y * d2y)
    c = (((o1 > tol1) & (o2 < -tol1)) | ((o1 < -tol1) & (o2 > tol1))) & \
        (((o3 > tol2) & (o4 < -tol2)) | ((o3 < -tol2) & (o4 > tol2)))
    return c & ~same


def cell_boxes(A, B, cell, lo0, lo1, nx, ny):
    """engine/charts.py:556-559: clamped cell ranges [x0, x1] x [y0, y1]."""
    box = np.empty((len(A), 4), np.int64)
    for i in range(len(A)):
        x0 = int((min(A[i, 0], B[i, 0]) - lo0) / cell); x1 = int((max(A[i, 0], B[i, 0]) - lo0) / cell)
        y0 = int((min(A[i, 1], B[i, 1]) - lo1) / cell); y1 = int((max(A[i, 1], B[i, 1]) - lo1) / cell)
        box[i] = (max(x0, 0), min(x1, nx - 1), max(y0, 0), min(y1, ny - 1))
    return box


def seg_intersections_cells(A, B, cell, lo, nx, ny, max_report):
    """engine/charts.py:547-593 as written: per-cell pair loops, early stop."""
    A = np.asarray(A, np.float64); B = np.asarray(B, np.float64)
    box = cell_boxes(A, B, cell, float(lo[0]), float(lo[1]), nx, ny)
    items = [[] for _ in range(nx * ny)]
    for i in range(len(A)):
        for gx in range(box[i, 0], box[i, 1] + 1):
            for gy in range(box[i, 2], box[i, 3] + 1):
                items[gy * nx + gx].append(i)
    hits = 0
    for lst in items:
        for p in range(len(lst)):
            i = lst[p]
            for q in range(p + 1, len(lst)):
                j = lst[q]
                if cross(A[i].tolist(), B[i].tolist(), A[j].tolist(), B[j].tolist()):
                    hits += 1
                    if hits >= max_report:
                        return hits
    return hits


def seg_intersections_pairs(A, B, cell, lo, nx, ny, max_report):
    """The same count from all pairs: crossing pairs weighted by shared cells."""
    A = np.asarray(A, np.float64); B = np.asarray(B, np.float64)
    box = cell_boxes(A, B, cell, float(lo[0]), float(lo[1]), nx, ny)
    c = np.triu(cross_matrix(A, B), 1)
    i, j = np.nonzero(c)
    ox = np.minimum(box[i, 1], box[j, 1]) - np.maximum(box[i, 0], box[j, 0]) + 1
    oy = np.minimum(box[i, 3], box[j, 3]) - np.maximum(box[i, 2], box[j, 2]) + 1
    total = int((np.maximum(ox, 0) * np.maximum(oy, 0)).sum())
    return min(total, max(int(max_report), 1)) if total else 0


def chart_grid(U, A, B):
    """engine/charts.py:601-607: lo, cell, nx, ny of one chart."""
    lo = U.min(0)
    ext = U.max(0) - lo
    L = np.linalg.norm(B - A, axis=1)
    cell = max(float(np.median(L)) * 4, float(ext.max()) / 512, 1e-30)
    nx = int(ext[0] / cell) + 1
    ny = int(ext[1] / cell) + 1
    return lo, cell, nx, ny


def boundary_intersections(U, T, max_report=1000, loops=False):
    """engine/charts.py:596-608 (ValueError for non-finite UVs, like the
    reference's int() of a non-finite grid size)."""
    U = np.asarray(U, np.float64).reshape(-1, 2)
    bi, bj = boundary_edges_oriented(T)
    if len(bi) < 3:
        return 0
    if not np.isfinite(U).all():
        raise ValueError("non-finite UVs")
    A = U[bi]; B = U[bj]
    lo, cell, nx, ny = chart_grid(U, A, B)
    f = seg_intersections_cells if loops else seg_intersections_pairs
    return int(f(A, B, cell, lo, nx, ny, max_report))


def hit(A, B):
    """engine/hier.py:227-266 (_hit): True if any two segments cross. The
    reference's grid only selects which pairs it tests; every crossing pair
    shares a cell, so the result is the same over all pairs."""
    A = np.asarray(A, np.float64); B = np.asarray(B, np.float64)
    if len(A) < 2:
        return False
    return bool(np.triu(cross_matrix(A, B), 1).any())


def _chart_hit(UV, ba, bb, ext_check=True):
    """engine/hier.py:334-352 (chart_checks: extent check) or 206-222
    (charts_collide: none) for one chart's segments."""
    if len(ba) < 3:
        return False
    A = UV[ba]; B = UV[bb]
    lo0 = min(A[:, 0].min(), B[:, 0].min()); hi0 = max(A[:, 0].max(), B[:, 0].max())
    lo1 = min(A[:, 1].min(), B[:, 1].min()); hi1 = max(A[:, 1].max(), B[:, 1].max())
    ext = max(hi0 - lo0, hi1 - lo1)
    if ext_check and not (ext < 1e300):
        return True
    return hit(A, B)


def boundary_directed(F, FF, faces, loc, chart, CV):
    """engine/hier.py:158-180 (loops over faces and corners)."""
    isb = _isb(F, FF, faces, loc, chart, CV)
    ba, bb = [], []
    for i in range(len(faces)):
        for k in range(3):
            if isb[i][k]:
                ba.append(CV[i][k]); bb.append(CV[i][(k + 1) % 3])
    return np.array(ba, np.int64), np.array(bb, np.int64)


def _isb(F, FF, faces, loc, chart, CV):
    isb = []
    for i, f in enumerate(faces):
        row = []
        for k in range(3):
            g = FF[f][k]
            b = True
            if g >= 0:
                j = loc[g]
                if j >= 0 and chart[j] == chart[i]:
                    a = F[f][k]
                    for kk in range(3):
                        if F[g][kk] == a:
                            if CV[j][kk] == CV[i][k]:
                                b = False
                            break
            row.append(b)
        isb.append(row)
    return isb


def charts_collide(CV, UV, chart, nchart, nv):
    """engine/hier.py:183-225."""
    CV = np.asarray(CV, np.int64); UV = np.asarray(UV, np.float64)
    keys = set()
    for i in range(len(CV)):
        for k in range(3):
            keys.add(int(CV[i, k]) * nv + int(CV[i, (k + 1) % 3]))
    segs = [[] for _ in range(nchart)]
    for i in range(len(CV)):
        for k in range(3):
            a, b = int(CV[i, k]), int(CV[i, (k + 1) % 3])
            if b * nv + a not in keys:
                segs[int(chart[i])].append((a, b))
    out = np.zeros(nchart, bool)
    for c in range(nchart):
        if segs[c]:
            s = np.array(segs[c], np.int64)
            out[c] = _chart_hit(UV, s[:, 0], s[:, 1], ext_check=False)
    return out


def _find(p, x):
    r = x
    while p[r] != r:
        r = p[r]
    while p[x] != r:
        nx = p[x]; p[x] = r; x = nx
    return r


def chart_checks(F, FF, faces, loc, chart, CV, UV, nchart, nv):
    """engine/hier.py:269-353 -> (collide, chi, loops), sequential loops."""
    F = np.asarray(F, np.int64).tolist(); FF = np.asarray(FF, np.int64).tolist()
    faces = np.asarray(faces, np.int64).tolist(); loc = np.asarray(loc, np.int64).tolist()
    chart = np.asarray(chart, np.int64).tolist(); CVa = np.asarray(CV, np.int64); CV = CVa.tolist()
    UV = np.asarray(UV, np.float64)
    n = len(faces)
    isb = _isb(F, FF, faces, loc, chart, CV)
    Fc = [0] * nchart; nb_c = [0] * nchart
    for i in range(n):
        Fc[chart[i]] += 1
        nb_c[chart[i]] += sum(isb[i])
    vchart = [-1] * nv
    for i in range(n):
        for k in range(3):
            vchart[CV[i][k]] = chart[i]
    Vc = [0] * nchart
    for v in range(nv):
        if vchart[v] >= 0:
            Vc[vchart[v]] += 1
    chi = np.array([Vc[c] - (3 * Fc[c] + nb_c[c]) // 2 + Fc[c] for c in range(nchart)], np.int64)
    segs = [[] for _ in range(nchart)]
    ba, bb = [], []
    for i in range(n):
        for k in range(3):
            if isb[i][k]:
                segs[chart[i]].append((CV[i][k], CV[i][(k + 1) % 3]))
    for c in range(nchart):
        for a, b in segs[c]:
            ba.append(a); bb.append(b)
    p = list(range(nv))
    for a, b in zip(ba, bb):
        ra = _find(p, a); rb = _find(p, b)
        if ra != rb:
            p[rb] = ra
    loops = np.zeros(nchart, np.int64)
    seen = [False] * nv
    for a, b in zip(ba, bb):
        for v in (a, b):
            if not seen[v]:
                seen[v] = True
                if _find(p, v) == v:
                    loops[vchart[v]] += 1
    collide = np.zeros(nchart, bool)
    for c in range(nchart):
        if len(segs[c]) >= 3:
            s = np.array(segs[c], np.int64)
            collide[c] = _chart_hit(UV, s[:, 0], s[:, 1])
    return collide, chi, loops
