"""Oracle for exact UV validation and UV metrics (test infrastructure only).

Vectorised numpy restatement of engine/validate.py and the parts of
engine/metrics.py it uses. Every FP64 operation follows the reference's
order (no fused multiply-add; numpy's left-to-right sums), so verdicts are
bit-exact. Candidate triangle pairs come from a uniform grid over the real
bounding boxes: the tolerant and strict predicates are only true for
triangles whose bounding boxes intersect, so any candidate set that holds
every such pair gives the reference's flags (engine/validate.py:95-136 tests
a superset of them). The gutter uses scipy.ndimage.distance_transform_edt,
the reference's own dependency (engine/metrics.py:351-358).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ULP = 2.0 ** -24
_CLIB = None


def clib():
    """The C restatement of the reference's serial loops (oracle/c/uva_oracle.c)."""
    global _CLIB
    if _CLIB is None:
        from oracle import build_oracle
        lib = C.CDLL(build_oracle.build())
        vp = C.c_void_p
        lib.uvo_overlaps.argtypes = [vp, vp, vp, C.c_int64, C.c_int64, C.c_double, C.c_int, vp]
        lib.uvo_overlaps.restype = C.c_int64
        lib.uvo_overlaps_band.argtypes = [vp, vp, vp, C.c_int64, C.c_int64, C.c_double, C.c_int, C.c_int64,
                                          C.c_int64, vp]
        lib.uvo_overlaps_band.restype = C.c_int64
        lib.uvo_raster_labels.argtypes = [vp, vp, vp, C.c_int64, C.c_int64, vp]
        lib.uvo_raster_labels.restype = None
        lib.uvo_raster_counts.argtypes = [vp, vp, C.c_int64, C.c_int64, vp]
        lib.uvo_raster_counts.restype = None
        lib.uvo_pack_raster.argtypes = [vp, vp, C.c_int64, C.c_int64, C.c_int64, vp]
        lib.uvo_pack_raster.restype = None
        lib.uvo_pack_try.argtypes = [C.c_int64, C.c_int64, C.c_int64] + [vp] * 11
        lib.uvo_pack_try.restype = C.c_int64
        _CLIB = lib
    return _CLIB


def _p(a):
    return C.c_void_p(a.ctypes.data)


def overlaps_c(U, F, skip, G, rel=1e-6, strict=False, band=None):
    """engine/validate.py:95-136 / :258-300 exactly as the reference loops
    (grid G, serial binning), in C. Returns (flags, tested cell-box pairs).
    band: (lo, hi) cell rows: only the pairs whose first shared cell lies in
    those rows (one shard of a sharded validation)."""
    U = np.ascontiguousarray(U, np.float64)
    F = np.ascontiguousarray(F, np.int64)
    sk = np.ascontiguousarray(skip, np.uint8)
    flag = np.zeros(len(F), np.uint8)
    lo, hi = (0, int(G)) if band is None else (int(band[0]), int(band[1]))
    n = clib().uvo_overlaps_band(_p(U), _p(F), _p(sk), len(F), int(G), float(rel), 1 if strict else 0, lo, hi,
                                 _p(flag))
    return flag.astype(bool), int(n)


# ------------------------------------------------------------------ predicates
def orient(ax, ay, bx, by, cx, cy):
    """engine/validate.py:21-22."""
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)


def strict_inside(px, py, ax, ay, bx, by, cx, cy, rel):
    """engine/validate.py:33-45."""
    l = np.maximum((bx - ax) ** 2 + (by - ay) ** 2, np.maximum((cx - bx) ** 2 + (cy - by) ** 2,
                                                              (ax - cx) ** 2 + (ay - cy) ** 2))
    eps = np.maximum(rel * l, 4.0 * ULP * np.sqrt(l)) if rel > 0 else np.zeros_like(l)
    d1 = orient(ax, ay, bx, by, px, py)
    d2 = orient(bx, by, cx, cy, px, py)
    d3 = orient(cx, cy, ax, ay, px, py)
    return ((d1 > eps) & (d2 > eps) & (d3 > eps)) | ((d1 < -eps) & (d2 < -eps) & (d3 < -eps))


def proper_cross(ax, ay, bx, by, cx, cy, dx, dy, rel):
    """engine/validate.py:48-54."""
    l1 = (bx - ax) ** 2 + (by - ay) ** 2
    l2 = (dx - cx) ** 2 + (dy - cy) ** 2
    e1 = np.maximum(rel * l1, 4.0 * ULP * np.sqrt(l1))
    e2 = np.maximum(rel * l2, 4.0 * ULP * np.sqrt(l2))
    o1 = orient(ax, ay, bx, by, cx, cy)
    o2 = orient(ax, ay, bx, by, dx, dy)
    o3 = orient(cx, cy, dx, dy, ax, ay)
    o4 = orient(cx, cy, dx, dy, bx, by)
    return (((o1 > e1) & (o2 < -e1)) | ((o1 < -e1) & (o2 > e1))) & (((o3 > e2) & (o4 < -e2)) | ((o3 < -e2) & (o4 > e2)))


def tri_overlap(U, F, S, T, rel, strict=False):
    """engine/validate.py:57-91 (tolerant) and :232-255 (strict), evaluated
    for the triangle pairs (S[k], T[k]). Early returns become masks."""
    a = U[F[S]]          # (k,3,2)
    b = U[F[T]]
    same = (a[:, :, None, 0] == b[:, None, :, 0]) & (a[:, :, None, 1] == b[:, None, :, 1])   # (k,3,3)
    shared = same.any(2).sum(1)
    live = shared != 3
    res = np.zeros(len(S), bool)
    for i in range(3):
        p0, p1 = i, (i + 1) % 3
        for j in range(3):
            q0, q1 = j, (j + 1) % 3
            sk = same[:, p0, q0] | same[:, p0, q1] | same[:, p1, q0] | same[:, p1, q1]
            A, B, C, D = a[:, p0], a[:, p1], b[:, q0], b[:, q1]
            if strict:
                o1 = orient(A[:, 0], A[:, 1], B[:, 0], B[:, 1], C[:, 0], C[:, 1])
                o2 = orient(A[:, 0], A[:, 1], B[:, 0], B[:, 1], D[:, 0], D[:, 1])
                o3 = orient(C[:, 0], C[:, 1], D[:, 0], D[:, 1], A[:, 0], A[:, 1])
                o4 = orient(C[:, 0], C[:, 1], D[:, 0], D[:, 1], B[:, 0], B[:, 1])
                hit = (o1 * o2 < 0) & (o3 * o4 < 0)
            else:
                hit = proper_cross(A[:, 0], A[:, 1], B[:, 0], B[:, 1], C[:, 0], C[:, 1], D[:, 0], D[:, 1], rel)
            res |= live & ~sk & hit
    if strict:
        return res
    for i in range(3):
        ns = ~same[:, i, :].any(1)
        res |= live & ns & strict_inside(a[:, i, 0], a[:, i, 1], b[:, 0, 0], b[:, 0, 1], b[:, 1, 0], b[:, 1, 1],
                                         b[:, 2, 0], b[:, 2, 1], rel)
        ns = ~same[:, :, i].any(1)
        res |= live & ns & strict_inside(b[:, i, 0], b[:, i, 1], a[:, 0, 0], a[:, 0, 1], a[:, 1, 0], a[:, 1, 1],
                                         a[:, 2, 0], a[:, 2, 1], rel)
    ca = ((a[:, 0] + a[:, 1]) + a[:, 2]) / 3.0
    cb = ((b[:, 0] + b[:, 1]) + b[:, 2]) / 3.0
    res |= live & strict_inside(ca[:, 0], ca[:, 1], b[:, 0, 0], b[:, 0, 1], b[:, 1, 0], b[:, 1, 1], b[:, 2, 0], b[:, 2, 1], rel)
    res |= live & strict_inside(cb[:, 0], cb[:, 1], a[:, 0, 0], a[:, 0, 1], a[:, 1, 0], a[:, 1, 1], a[:, 2, 0], a[:, 2, 1], rel)
    return res


def bbox_pairs(U, F, skip, max_cells=64):
    """Unordered pairs (s < t) of non-skipped triangles whose closed FP64
    bounding boxes intersect. Triangles covering more than ``max_cells`` grid
    cells are paired with every triangle by a direct box test."""
    idx = np.flatnonzero(~skip)
    if len(idx) < 2:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    u = U[F[idx]]
    lo = u.min(1)
    hi = u.max(1)
    org = lo.min(0)
    span = np.maximum(hi.max(0) - org, 1e-300)
    ext = np.maximum(np.median(hi - lo, 0), span / 4096)
    G = np.clip((span / ext).astype(np.int64), 1, 4096)
    c0 = np.clip(((lo - org) / span * G).astype(np.int64), 0, G - 1)
    c1 = np.clip(((hi - org) / span * G).astype(np.int64), 0, G - 1)
    nx = c1[:, 0] - c0[:, 0] + 1
    ny = c1[:, 1] - c0[:, 1] + 1
    cnt = nx * ny
    big = np.flatnonzero(cnt > max_cells)
    small = np.flatnonzero(cnt <= max_cells)
    S, T = [], []
    # small triangles: shared grid cells
    c = cnt[small]
    rep = np.repeat(small, c)
    k = np.arange(len(rep)) - np.repeat(np.cumsum(c) - c, c)
    cx = c0[rep, 0] + k % nx[rep]
    cy = c0[rep, 1] + k // nx[rep]
    cell = cy * G[0] + cx
    o = np.argsort(cell, kind="stable")
    cell = cell[o]
    item = rep[o]
    if len(cell):
        starts = np.flatnonzero(np.r_[True, cell[1:] != cell[:-1]])
        sizes = np.diff(np.r_[starts, len(cell)])
        for sz in np.unique(sizes):
            if sz < 2:
                continue
            st = starts[sizes == sz]
            ii, jj = np.triu_indices(sz, 1)
            S.append(item[st[:, None] + ii[None, :]].ravel())
            T.append(item[st[:, None] + jj[None, :]].ravel())
    # big triangles: direct box test against everything
    for bi in big:
        hit = (lo[:, 0] <= hi[bi, 0]) & (lo[bi, 0] <= hi[:, 0]) & (lo[:, 1] <= hi[bi, 1]) & (lo[bi, 1] <= hi[:, 1])
        hit[bi] = False
        other = np.flatnonzero(hit)
        S.append(np.full(len(other), bi)); T.append(other)
    if not S:
        return np.empty(0, np.int64), np.empty(0, np.int64)
    S = np.concatenate(S); T = np.concatenate(T)
    a = np.minimum(S, T); b = np.maximum(S, T)
    key = np.unique(a * len(idx) + b)
    a = key // len(idx); b = key % len(idx)
    keep = (lo[a, 0] <= hi[b, 0]) & (lo[b, 0] <= hi[a, 0]) & (lo[a, 1] <= hi[b, 1]) & (lo[b, 1] <= hi[a, 1])
    return idx[a[keep]], idx[b[keep]]


def count_bbox_pairs(U, F, skip):
    """Unordered non-skipped pairs whose closed FP64 boxes intersect (P_aabb)."""
    return len(bbox_pairs(U, F, skip)[0])


def overlaps(U, F, skip, rel=1e-6, strict=False, chunk=1 << 20):
    """Per-triangle flags of engine/validate.py:95-136 (_overlaps) or
    :258-300 (_overlaps_strict)."""
    S, T = bbox_pairs(U, F, skip)
    flag = np.zeros(len(F), bool)
    for c in range(0, len(S), chunk):
        s, t = S[c:c + chunk], T[c:c + chunk]
        hit = tri_overlap(U, F, s, t, rel, strict)
        flag[s[hit]] = True
        flag[t[hit]] = True
    return flag, len(S)


# ------------------------------------------------------------------ islands
def uv_islands(faces, n_vertices, uv=None, vertices=None):
    """engine/metrics.py:91-103: weld vertices with identical float32
    (position, uv) bytes, label faces by connected components. Labels are
    numbered by the smallest face index of each island (the partition is the
    reference's; its label numbering depends on union order)."""
    faces = np.asarray(faces, np.int64)
    if uv is not None and vertices is not None:
        key = np.concatenate([np.asarray(vertices, np.float32), np.asarray(uv, np.float32)], 1)
        key = np.ascontiguousarray(key).view(np.dtype((np.void, 20))).reshape(-1)
        _, inv = np.unique(key, return_inverse=True)
        faces = inv.reshape(-1)[faces]
        n_vertices = int(inv.max()) + 1 if len(inv) else 0
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg
    m = len(faces)
    if m == 0:
        return np.zeros(0, np.int32), 0
    rows = np.repeat(np.arange(m), 3)
    G = sp.csr_matrix((np.ones(3 * m), (rows, faces.ravel())), shape=(m, n_vertices))
    A = (G @ G.T).tocsr()
    n, lab = cg.connected_components(A, directed=False)
    first = np.full(n, m, np.int64)
    np.minimum.at(first, lab, np.arange(m))
    rank = np.empty(n, np.int64)
    rank[np.argsort(first)] = np.arange(n)
    return rank[lab].astype(np.int32), int(n)


def same_partition(a, b):
    """True if two labelings define the same partition."""
    a = np.asarray(a); b = np.asarray(b)
    if a.shape != b.shape:
        return False
    pairs = np.unique(np.stack([a, b], 1), axis=0)
    return len(pairs) == len(np.unique(a)) == len(np.unique(b))


# ------------------------------------------------------------------ gutter
def raster_labels(uv, faces, lab_of_face, res):
    """engine/metrics.py:315-345: conservative raster, the last triangle in
    index order wins each texel (C loop, same order as the reference)."""
    uv = np.ascontiguousarray(uv, np.float64)
    F = np.ascontiguousarray(faces, np.int64)
    lab = np.ascontiguousarray(lab_of_face, np.int32)
    img = np.full((res, res), -1, np.int32)
    clib().uvo_raster_labels(_p(uv), _p(F), _p(lab), len(F), int(res), _p(img))
    return img


def raster_counts(uv, faces, res):
    """engine/metrics.py:13-54 (top-left rule, uint8 saturating counts)."""
    uv = np.ascontiguousarray(uv, np.float64)
    F = np.ascontiguousarray(faces, np.int64)
    counts = np.zeros((res, res), np.uint8)
    clib().uvo_raster_counts(_p(uv), _p(F), len(F), int(res), _p(counts))
    return counts


def raster_labels_numpy(uv, faces, lab_of_face, res):
    """Vectorised numpy version of raster_labels (cross-check of the C loop)."""
    uv = np.asarray(uv, np.float64)
    F = np.asarray(faces, np.int64)
    img_t = np.full(res * res, -1, np.int64)
    x = uv[F, 0] * res
    y = uv[F, 1] * res
    area = (x[:, 1] - x[:, 0]) * (y[:, 2] - y[:, 0]) - (x[:, 2] - x[:, 0]) * (y[:, 1] - y[:, 0])
    neg = area < 0
    x[neg, 1], x[neg, 2] = x[neg, 2].copy(), x[neg, 1].copy()
    y[neg, 1], y[neg, 2] = y[neg, 2].copy(), y[neg, 1].copy()
    with np.errstate(invalid="ignore"):
        minx = np.maximum(np.floor(x.min(1)), 0)
        maxx = np.minimum(np.floor(x.max(1)), res - 1)
        miny = np.maximum(np.floor(y.min(1)), 0)
        maxy = np.minimum(np.floor(y.max(1)), res - 1)
    ok = np.isfinite(minx) & np.isfinite(maxx) & np.isfinite(miny) & np.isfinite(maxy) & (minx <= maxx) & (miny <= maxy)
    tris = np.flatnonzero(ok)
    minx = minx[tris].astype(np.int64); maxx = maxx[tris].astype(np.int64)
    miny = miny[tris].astype(np.int64); maxy = maxy[tris].astype(np.int64)
    nx = maxx - minx + 1
    cnt = nx * (maxy - miny + 1)
    ex = np.stack([x[:, 1] - x[:, 0], x[:, 2] - x[:, 1], x[:, 0] - x[:, 2]], 1)[tris]
    ey = np.stack([y[:, 1] - y[:, 0], y[:, 2] - y[:, 1], y[:, 0] - y[:, 2]], 1)[tris]
    ox = x[tris]; oy = y[tris]
    L = np.sqrt(ex ** 2 + ey ** 2)
    step = 1 << 22
    csum = np.cumsum(cnt)
    start = 0
    while start < len(tris):
        stop = int(np.searchsorted(csum, (csum[start - 1] if start else 0) + step, side="right"))
        stop = max(stop, start + 1)
        sl = slice(start, stop)
        c = cnt[sl]
        rep = np.repeat(np.arange(start, stop), c)
        k = np.arange(len(rep)) - np.repeat(np.cumsum(c) - c, c)
        px = minx[rep] + k % nx[rep]
        py = miny[rep] + k // nx[rep]
        cx = px + 0.5
        cy = py + 0.5
        inside = np.ones(len(rep), bool)
        for e in range(3):
            ev = ex[rep, e] * (cy - oy[rep, e]) - ey[rep, e] * (cx - ox[rep, e])
            inside &= ~(ev < -0.7072 * L[rep, e])
        np.maximum.at(img_t, (py * res + px)[inside], tris[rep[inside]])
        start = stop
    lab = np.asarray(lab_of_face, np.int64)
    img = np.where(img_t >= 0, lab[np.maximum(img_t, 0)], -1).astype(np.int32)
    return img.reshape(res, res)


def min_gutter(uv, faces, islands, res=4096):
    """engine/metrics.py:348-373."""
    from scipy import ndimage
    img = raster_labels(uv, faces, islands, res)
    empty = img < 0
    if empty.all() or not empty.any():
        return float("nan"), img
    d, (iy, ix) = ndimage.distance_transform_edt(empty, return_indices=True)
    near = img[iy, ix]
    touch = ((img[:, 1:] >= 0) & (img[:, :-1] >= 0) & (img[:, 1:] != img[:, :-1])).any() or \
        ((img[1:, :] >= 0) & (img[:-1, :] >= 0) & (img[1:, :] != img[:-1, :])).any()
    if touch:
        return 0.0, img
    dif_h = near[:, 1:] != near[:, :-1]
    dif_v = near[1:, :] != near[:-1, :]
    g = np.inf
    if dif_h.any():
        g = min(g, float((d[:, 1:] + d[:, :-1])[dif_h].min()))
    if dif_v.any():
        g = min(g, float((d[1:, :] + d[:-1, :])[dif_v].min()))
    return max(g - 1.0, 0.0), img


# ------------------------------------------------------------------ report
def validate_uvs(v, f, uv, atlas=4096, padding=None, gutter=True, rel=1e-6, count_pairs=True):
    """engine/validate.py:139-209 (without the preservation inputs).
    Returns (report, problems mask, extras). ``count_pairs`` adds the number
    of candidate pairs with intersecting boxes (the pairs/s denominator; not
    part of the reference's work)."""
    v = np.asarray(v, np.float64)
    f = np.asarray(f, np.int64)
    U = np.asarray(uv, np.float32).astype(np.float64)
    rep = {}
    rep["non_finite_uv"] = int((~np.isfinite(U)).any(1).sum())
    with np.errstate(invalid="ignore"):
        rep["uv_outside_unit_square"] = int(((U < 0) | (U > 1)).any(1).sum())
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    a3 = 0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1)
    u = U[f]
    with np.errstate(invalid="ignore", over="ignore"):
        sa = 0.5 * ((u[:, 1, 0] - u[:, 0, 0]) * (u[:, 2, 1] - u[:, 0, 1]) - (u[:, 2, 0] - u[:, 0, 0]) * (u[:, 1, 1] - u[:, 0, 1]))
        edge = np.maximum(np.maximum(np.linalg.norm(u[:, 1] - u[:, 0], axis=1), np.linalg.norm(u[:, 2] - u[:, 1], axis=1)),
                          np.linalg.norm(u[:, 0] - u[:, 2], axis=1))
        sliver = np.abs(sa) < 2.0 ** -24 * np.maximum(edge, 2.0 ** -24)
    has3d = a3 > 1e-14 * max(float(a3.max()) if len(a3) else 0.0, 1e-30)
    rep["degenerate_uv_triangles"] = int((has3d & (sa == 0)).sum())
    rep["sub_float32_slivers"] = int((has3d & sliver).sum())
    isl, n = uv_islands(f, len(v), U, v)
    w = np.abs(sa)
    pos = np.bincount(isl, weights=np.where(sa > 0, w, 0), minlength=n)
    neg = np.bincount(isl, weights=np.where(sa < 0, w, 0), minlength=n)
    dom = np.where(pos >= neg, 1.0, -1.0)
    flipped = has3d & ~sliver & (np.sign(sa) != dom[isl]) & (sa != 0)
    rep["flipped_triangles"] = int(flipped.sum())
    rep["mirrored_islands"] = int((neg > pos).sum())
    rep["islands"] = int(n)
    skip = ~has3d | sliver | ~np.isfinite(sa)
    G = int(np.clip(np.sqrt(len(f)) / 2, 64, 4096))
    ov, _ = overlaps_c(U, f, skip, G, rel)
    npairs = count_bbox_pairs(U, f, skip) if count_pairs else None
    rep["overlapping_triangles_exact"] = int(ov.sum())
    ovs, _ = overlaps_c(U, f, skip, G, 0.0, strict=True)
    rep["float32_contacts"] = int((ovs & ~ov).sum())
    if ov.any():
        rep["islands_with_overlap"] = int(len(np.unique(isl[ov])))
    if gutter:
        res = min(atlas, 8192)
        g, _ = min_gutter(U, f, isl, res)
        rep["min_gutter_texels"] = float(g * atlas / res)
        if padding is not None:
            rep["gutter_ok"] = bool(rep["min_gutter_texels"] >= padding - 1e-6)
    problems = ov | flipped
    bad = rep["non_finite_uv"] + rep["uv_outside_unit_square"] + rep["flipped_triangles"] + rep["overlapping_triangles_exact"]
    if gutter and padding is not None and not rep.get("gutter_ok", True):
        bad += 1
    rep["valid"] = bool(bad == 0)
    extras = {"ov": ov, "ov_strict": ovs, "flipped": flipped, "islands": isl, "pairs": npairs, "skip": skip}
    return rep, problems, extras


def chart_overlaps(U, T):
    """engine/validate.py:212-226."""
    U = np.asarray(U, np.float64)
    T = np.asarray(T, np.int64)
    if len(T) < 2:
        return np.zeros(len(T), bool)
    lo = U.min(0)
    ext = float((U.max(0) - lo).max())
    if not np.isfinite(ext) or ext <= 0:
        return np.zeros(len(T), bool)
    Un = (U - lo) / ext * 0.999999
    u = Un[T]
    sa = 0.5 * ((u[:, 1, 0] - u[:, 0, 0]) * (u[:, 2, 1] - u[:, 0, 1]) - (u[:, 2, 0] - u[:, 0, 0]) * (u[:, 1, 1] - u[:, 0, 1]))
    skip = np.abs(sa) <= 1e-14
    return overlaps(Un, T, skip, 1e-6)[0]
