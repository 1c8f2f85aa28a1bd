"""Oracle for the per-chart overlap checks (test infrastructure only).

Pure-Python restatement of engine/overlapfix.py of the reference:
_raster_all / overlapping_triangles (:173-224), _raster_pair /
raster_overlap (:135-170, 263-275), _boundary_with_faces (:16-41) and
_first_hit / collision (:44-84, 283-296), as serial loops in the reference's
order (small cases). Pinned against golden_overlap.npz, made by running the
reference itself (tests/golden/make_golden_overlap.py).
"""
from __future__ import annotations

import math

import numpy as np

from oracle import segments as OS


def _texels(uv, tri, res):
    """Texel centres triangle `tri` covers, in the reference's scan order
    (top-left rule, engine/overlapfix.py:144-168)."""
    a, b, c = tri
    x0, y0 = uv[a][0] * res, uv[a][1] * res
    x1, y1 = uv[b][0] * res, uv[b][1] * res
    x2, y2 = uv[c][0] * res, uv[c][1] * res
    ar = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0)
    if ar == 0.0:
        return
    if ar < 0:
        x1, y1, x2, y2 = x2, y2, x1, y1
    minx = max(int(math.floor(min(x0, min(x1, x2)) - 0.5)), 0)
    maxx = min(int(math.ceil(max(x0, max(x1, x2)) - 0.5)), res - 1)
    miny = max(int(math.floor(min(y0, min(y1, y2)) - 0.5)), 0)
    maxy = min(int(math.ceil(max(y0, max(y1, y2)) - 0.5)), res - 1)
    ex = (x1 - x0, x2 - x1, x0 - x2); ey = (y1 - y0, y2 - y1, y0 - y2)
    ox = (x0, x1, x2); oy = (y0, y1, y2)
    for py in range(miny, maxy + 1):
        cy = py + 0.5
        for px in range(minx, maxx + 1):
            cx = px + 0.5
            inside = True
            for k in range(3):
                e = ex[k] * (cy - oy[k]) - ey[k] * (cx - ox[k])
                if e < 0 or (e == 0 and not ((ey[k] == 0 and ex[k] < 0) or ey[k] > 0)):
                    inside = False
                    break
            if inside:
                yield py, px


def _normalised(U):
    U = np.asarray(U, np.float64).reshape(-1, 2)
    lo = U.min(0)
    ext = float((U.max(0) - lo).max())
    if not np.isfinite(ext) or ext <= 0:
        return None
    return ((U - lo) / ext * 0.999).tolist()


def overlapping_triangles(U, T, res=None):
    T = np.asarray(T, np.int64).reshape(-1, 3)
    bad = np.zeros(len(T), np.bool_)
    if len(T) < 2:
        return bad
    uv = _normalised(U)
    if uv is None:
        return bad
    if res is None:
        res = int(np.clip(np.sqrt(len(T)) * 2.5, 64, 3072))
    owner = {}
    for t, tri in enumerate(T.tolist()):
        for key in _texels(uv, tri, res):
            o = owner.get(key, -1)
            if o >= 0:
                bad[o] = True
                bad[t] = True
            else:
                owner[key] = t
    return bad


def raster_overlap(U, T, res=None):
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if len(T) < 2:
        return None
    uv = _normalised(U)
    if uv is None:
        return None
    if res is None:
        res = int(np.clip(np.sqrt(len(T)) * 2.0, 64, 2048))
    owner = {}
    for t, tri in enumerate(T.tolist()):
        for key in _texels(uv, tri, res):
            o = owner.get(key, -1)
            if o >= 0:
                return o, t
            owner[key] = t
    return None


def boundary_with_faces(T):
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if len(T) == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64)
    n = int(T.max()) + 1
    keys = set()
    for f in range(len(T)):
        for k in range(3):
            keys.add(int(T[f, k]) * n + int(T[f, (k + 1) % 3]))
    a, b, fo = [], [], []
    for f in range(len(T)):
        for k in range(3):
            i, j = int(T[f, k]), int(T[f, (k + 1) % 3])
            if j * n + i in keys:
                continue
            a.append(i); b.append(j); fo.append(f)
    return np.array(a, np.int64), np.array(b, np.int64), np.array(fo, np.int64)


def first_hit(A, B, cell, lo, nx, ny):
    """engine/overlapfix.py:44-84: cells in order, pairs in item order."""
    box = OS.cell_boxes(A, B, cell, float(lo[0]), float(lo[1]), nx, ny)
    items = [[] for _ in range(nx * ny)]
    for i in range(len(A)):
        for gx in range(box[i, 0], box[i, 1] + 1):
            for gy in range(box[i, 2], box[i, 3] + 1):
                items[gy * nx + gx].append(i)
    for lst in items:
        for p in range(len(lst)):
            for q in range(p + 1, len(lst)):
                i, j = lst[p], lst[q]
                if OS.cross(A[i].tolist(), B[i].tolist(), A[j].tolist(), B[j].tolist()):
                    return i, j
    return -1, -1


def collision(U, T):
    U = np.asarray(U, np.float64).reshape(-1, 2)
    a, b, fo = boundary_with_faces(T)
    if len(a) < 3:
        return None
    if not np.isfinite(U).all():
        raise ValueError("non-finite UVs")
    A = U[a]; B = U[b]
    lo = U.min(0); ext = U.max(0) - lo
    L = np.linalg.norm(B - A, axis=1)
    cell = max(float(np.median(L)) * 4, float(ext.max()) / 1024, 1e-30)
    nx = int(ext[0] / cell) + 1; ny = int(ext[1] / cell) + 1
    i, j = first_hit(A, B, cell, lo, nx, ny)
    if i < 0:
        return None
    return int(fo[i]), int(fo[j])
