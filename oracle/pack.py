"""Oracle for the raster atlas packer (test infrastructure only).

CPU restatement of engine/pack.py: orientation to the minimum-area
rectangle (:19-48), conservative chart masks with a square gutter dilation
(:52-92, the raster loop in C: oracle/c/uva_oracle.c uvo_pack_raster), row
runs (:95-119), the greedy first fit of all charts with the free-run and
occupied-run tables (:123-156, :232-256, :312-359, in C: uvo_pack_try), the
masks of every (angle, quarter turn) with the two-orientation rule for tiny
islands (:373-388), the island orderings (:391-395), the bisection and
k-ary scale searches (:409-468) and pack() with its coarse-to-fine schedule
(:471-554). The maximal-contact placement (:169-220, :325-342) is not
restated: the reference runs it for no chart (CONTACT_MAX_CHARTS = 0).
Pinned against the reference's own outputs in tests/golden/golden_pack.npz.
"""
from __future__ import annotations

import time

import numpy as np

from oracle.validate import clib

ORDER_KEYS = ("area", "bbox", "height")
MANY_CHARTS = 1500


def _p(a):
    return a.ctypes.data


# ------------------------------------------------------------------ orientation
def min_area_rect_angle(U):
    """pack.py:19-37: the hull edge angle (mod 90 degrees, rounded to 9
    digits) whose rotation gives the smallest bounding rectangle."""
    from scipy.spatial import ConvexHull
    if len(U) < 3:
        return 0.0
    try:
        hull = U[ConvexHull(U).vertices]
    except Exception:  # noqa: BLE001 - degenerate input: no rotation, as the reference
        return 0.0
    e = np.roll(hull, -1, 0) - hull
    cands = np.unique(np.round(np.mod(np.arctan2(e[:, 1], e[:, 0]), np.pi / 2), 9))
    best_area, best_a = np.inf, 0.0
    for a in cands:
        c, s = np.cos(-a), np.sin(-a)
        Rh = hull @ np.array([[c, -s], [s, c]]).T
        ext = Rh.max(0) - Rh.min(0)
        if ext[0] * ext[1] < best_area - 1e-12:
            best_area, best_a = ext[0] * ext[1], a
    return best_a


def orient(U):
    """pack.py:40-48: rotate to the minimum-area rectangle, landscape, min 0."""
    a = min_area_rect_angle(U)
    c, s = np.cos(-a), np.sin(-a)
    V = U @ np.array([[c, -s], [s, c]]).T
    ext = V.max(0) - V.min(0)
    if ext[1] > ext[0]:
        V = V[:, ::-1] * np.array([1, -1])
    return V - V.min(0)


def rotated(U, a):
    """pack.py:365-370."""
    if a == 0.0:
        return U
    c, s = np.cos(a), np.sin(a)
    V = U @ np.array([[c, -s], [s, c]]).T
    return V - V.min(0)


def uv_area(U, T):
    """pack.py:570-572."""
    a, b, c = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
    return float(np.abs(0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1])
                               - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))).sum())


# ------------------------------------------------------------------ masks
def chart_mask(U, T, scale, pad):
    """pack.py:82-92: (h, w) uint8 mask of an oriented chart at `scale`
    texels per unit with a `pad`-texel border, dilated by `pad`."""
    V = np.ascontiguousarray(U * scale + pad, np.float64)
    w = int(np.ceil(V[:, 0].max() + pad)) + 1
    h = int(np.ceil(V[:, 1].max() + pad)) + 1
    m = np.zeros((h, w), np.uint8)
    T = np.ascontiguousarray(T, np.int64)
    clib().uvo_pack_raster(_p(V), _p(T), len(T), h, w, _p(m))
    if pad > 0:
        from scipy.ndimage import maximum_filter
        m = maximum_filter(m, size=2 * pad + 1, mode="constant", cval=0)
    return m


def intervals(mask):
    """pack.py:95-119: per row the runs of set cells (first, last) and the
    longest run; ptr: run offsets per row."""
    m = np.ascontiguousarray(mask, np.uint8).astype(bool)
    h, w = m.shape
    pm = np.zeros((h, w + 2), np.int8)
    pm[:, 1:-1] = m
    d = np.diff(pm, axis=1)
    rs, cs = np.nonzero(d == 1)       # run starts, row-major order
    _, ce = np.nonzero(d == -1)       # one past the run ends
    ptr = np.zeros(h + 1, np.int64)
    np.add.at(ptr, rs + 1, 1)
    ptr = np.cumsum(ptr)
    need = np.zeros(h, np.int64)
    np.maximum.at(need, rs, ce - cs)
    return ptr, cs.astype(np.int64), (ce - 1).astype(np.int64), need


def masks_at(Us, Ts, dens, s, pad, rot_set, angles=(0.0,)):
    """pack.py:373-388: per chart the masks of every (angle, quarter turn),
    k = angle_index * len(rot_set) + turn; tiny islands (under 400 cells)
    keep turns 0 and 1 at angle 0 only (None elsewhere)."""
    out = []
    for U, T, d in zip(Us, Ts, dens):
        ms = []
        for a in angles:
            m0 = chart_mask(rotated(U, a), T, s * d, pad)
            tiny = m0.shape[0] * m0.shape[1] < 400
            for r in rot_set:
                if tiny and (r >= 2 or a != 0.0):
                    ms.append(None)
                    continue
                ms.append(np.ascontiguousarray(np.rot90(m0, r)))
        out.append(ms)
    return out


def order_of(masks, ordering):
    """pack.py:391-400: charts by decreasing key (stable)."""
    m0 = [ms[0] for ms in masks]
    if ordering == "area":
        key = np.array([int(m.sum()) for m in m0])
    elif ordering == "bbox":
        key = np.array([m.shape[0] * m.shape[1] for m in m0])
    elif ordering == "height":
        key = np.array([min(m.shape) for m in m0])
    else:
        raise ValueError(f"unknown ordering {ordering!r}")
    return np.argsort(-key, kind="stable")


# ------------------------------------------------------------------ placement
def try_pack(masks, order, G):
    """pack.py:312-359 (first fit only): (placement list of (k, x, y), occ)
    or None when a chart fits nowhere."""
    nc = len(masks)
    nk = len(masks[0]) if nc else 0
    vh, vw, var_row, var_rp, ra, rb, need, rows = [], [], [0], [], [], [], [], []
    nrun = 0
    for ms in masks:
        for m in ms:
            if m is None:
                vh.append(0); vw.append(0); var_row.append(var_row[-1]); var_rp.append(np.array([nrun]))
                continue
            ptr, a, b, nd = intervals(m)
            vh.append(m.shape[0]); vw.append(m.shape[1]); var_row.append(var_row[-1] + m.shape[0])
            var_rp.append(ptr + nrun)
            ra.append(a); rb.append(b); need.append(nd)
            rows.append(np.argsort(-nd, kind="stable"))
            nrun += len(a)
    cat = lambda xs: np.ascontiguousarray(np.concatenate(xs), np.int64) if xs else np.zeros(1, np.int64)  # noqa: E731
    vh, vw = np.array(vh, np.int64), np.array(vw, np.int64)
    var_row, var_rp = np.array(var_row, np.int64), cat(var_rp)
    ra, rb, need, rows = cat(ra), cat(rb), cat(need), cat(rows)
    order = np.ascontiguousarray(order, np.int64)
    placement = np.full((max(nc, 1), 3), -1, np.int64)
    occ = np.zeros((G, G), np.uint8)
    rc = clib().uvo_pack_try(nc, nk, G, _p(order), _p(vh), _p(vw), _p(var_row), _p(var_rp), _p(ra), _p(rb),
                             _p(need), _p(rows), _p(placement), _p(occ))
    if rc != 0:
        return None
    return [tuple(int(v) for v in placement[i]) for i in range(nc)], occ


def attempt(Us, Ts, dens, G, pad, rot_set, s, ordering="area", angles=(0.0,)):
    """pack.py:398-402."""
    masks = masks_at(Us, Ts, dens, s, pad, rot_set, angles)
    res = try_pack(masks, order_of(masks, ordering), G)
    return None if res is None else (s, res, masks)


# ------------------------------------------------------------------ scale search
def search(attempt_fn, n, s, iters, tol=0.004, lo=0.0, hi=None, best=None, deadline=None):
    """pack.py:409-415: k-ary search from MANY_CHARTS islands, else bisection.
    attempt_fn(scale) -> result or None."""
    if n >= MANY_CHARTS:
        return search_kary(attempt_fn, s, iters, tol, lo, hi, best, deadline)
    return search_bisect(attempt_fn, s, iters, tol, lo, hi, best, deadline)


def search_kary(attempt_fn, s, iters, tol, lo, hi, best, deadline):
    """pack.py:418-445: four scales per round (tried one after another here:
    only which of them fit matters)."""
    k = 4
    for _ in range(max(2, int(np.ceil(iters / np.log2(k + 1))))):
        if hi is not None and lo > 0 and (hi - lo) / lo < tol:
            break
        if deadline is not None and best is not None and time.perf_counter() > deadline:
            break
        if lo == 0.0 and hi is None:
            cand = s * np.array([0.8, 0.9, 1.0, 1.1])[:k]
        elif hi is None:
            cand = lo * np.array([1.08, 1.17, 1.27, 1.4])[:k]
        elif lo == 0.0:
            cand = hi * np.array([0.55, 0.7, 0.8, 0.9])[:k]
        else:
            cand = np.linspace(lo, hi, k + 2)[1:-1]
        res = [attempt_fn(float(sc)) for sc in cand]
        for sc, r in zip(cand, res):
            if r is not None and sc > lo:
                best, lo = r, float(sc)
        fails = [float(sc) for sc, r in zip(cand, res) if r is None and sc > lo]
        if fails:
            hi = min(fails) if hi is None else min(hi, min(fails))
    return best, lo, hi


def search_bisect(attempt_fn, s, iters, tol, lo, hi, best, deadline):
    """pack.py:448-468: bracketing bisection; grows by 1.2 until a failure,
    shrinks by 0.8 until a success."""
    for _ in range(iters):
        if hi is not None and lo > 0 and (hi - lo) / lo < tol:
            break
        if deadline is not None and best is not None and time.perf_counter() > deadline:
            break
        r = attempt_fn(s)
        if r is not None:
            best, lo = r, s
        else:
            hi = s
        if hi is None:
            s *= 1.2
        elif lo == 0.0:
            s *= 0.8
        else:
            s = 0.5 * (lo + hi)
    return best, lo, hi


def rot_coords(V, rot, h, w):
    """pack.py:557-567."""
    x, y = V[:, 0], V[:, 1]
    rot %= 4
    if rot == 0:
        return np.stack([x, y], 1)
    if rot == 1:
        return np.stack([y, w - x], 1)
    if rot == 2:
        return np.stack([w - x, h - y], 1)
    return np.stack([h - y, x], 1)


def pack(charts, atlas=4096, padding=4, grid=None, rotations=4, density=None, iters=10, time_budget=None,
         orderings=("area", "bbox", "height"), angles=(0.0,), fine_attempts=8):
    """pack.py:471-554 (no log callback): (uvs, info)."""
    t0 = time.perf_counter()
    angles = tuple(float(a) for a in angles)
    deadline = None if not time_budget else t0 + float(time_budget)
    grid = grid or min(atlas, 2048)
    pad = int(np.ceil(padding * grid / atlas))
    n = len(charts)
    dens = np.ones(n) if density is None else np.asarray(density, float)
    Us = [orient(U) for U, _ in charts]
    Ts = [np.ascontiguousarray(T, np.int64) for _, T in charts]
    area = np.array([uv_area(U, T) * d * d for U, T, d in zip(Us, Ts, dens)])
    tot = max(area.sum(), 1e-30)
    rot_set = [0, 1, 2, 3][:max(1, rotations)]

    def at(G, p, o):
        return lambda sc: attempt(Us, Ts, dens, G, p, rot_set, sc, o, angles)

    best = None
    if grid >= 1024:
        g2 = grid // 2
        pad2 = max(1, int(np.ceil(padding * g2 / atlas)))
        b2, ordering = None, orderings[0]
        for o in orderings:
            if deadline is not None and b2 is not None and time.perf_counter() > t0 + 0.4 * float(time_budget):
                break
            s0 = b2[0] if b2 is not None else np.sqrt(0.62 * g2 * g2 / tot)
            bo, _, _ = search(at(g2, pad2, o), n, s0, iters, tol=0.01,
                              deadline=None if deadline is None else t0 + 0.6 * float(time_budget))
            if bo is not None and (b2 is None or bo[0] > b2[0]):
                b2, ordering = bo, o
        if b2 is not None:
            s0 = b2[0] * grid / g2 * 0.98
            r, used = None, 0
            for _ in range(4):
                r = attempt(Us, Ts, dens, grid, pad, rot_set, s0, ordering, angles)
                used += 1
                if r is not None:
                    break
                s0 *= 0.96
            if r is not None:
                lo_, hi_ = s0, s0 * 1.06
                for _ in range(8):
                    if (deadline is not None and time.perf_counter() > deadline) or used >= fine_attempts:
                        break
                    used += 1
                    r2 = attempt(Us, Ts, dens, grid, pad, rot_set, hi_, ordering, angles)
                    if r2 is None:
                        break
                    r, lo_, hi_ = r2, hi_, hi_ * 1.06
                best = r
                if fine_attempts - used > 0:
                    best, _, _ = search(at(grid, pad, ordering), n, 0.5 * (lo_ + hi_), min(3, fine_attempts - used),
                                        tol=0.006, lo=lo_, hi=hi_, best=r, deadline=deadline)
    if best is None:
        best, _, _ = search(at(grid, pad, "area"), n, np.sqrt(0.62 * grid * grid / tot), iters)
    if best is None:
        raise RuntimeError("packing failed: charts do not fit one page even at small scale")
    s, (placement, occ), masks = best
    nr = len(rot_set)
    uvs = []
    for i, (U, d) in enumerate(zip(Us, dens)):
        k, x, y = placement[i]
        ai, rot = k // nr, k % nr
        h0, w0 = masks[i][ai * nr].shape
        V = rotated(U, angles[ai]) * s * d + pad
        uvs.append((rot_coords(V, rot, h0, w0) + np.array([x, y])) / grid)
    info = {"texel_scale_grid": s, "texels_per_unit_atlas": s * atlas / grid, "grid": grid, "grid_padding": pad,
            "plan_occupancy": float(occ.mean()), "seconds": time.perf_counter() - t0}
    return uvs, info
