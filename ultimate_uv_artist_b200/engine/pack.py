"""Drop-in replacement of the reference's ``engine/pack.py``: the shape-exact
raster atlas packer.

``pack`` keeps the reference's signature, schedule and results
(engine/pack.py:471-554): charts are turned to their minimum-area rectangle
(:19-48, on the host), and every packing attempt at one texel scale runs on
the device in csrc/pack.cu — conservative chart masks with the gutter
dilation (:52-92), their row runs (:95-119), and the greedy first fit of all
charts over free-run tables in one cooperative launch (:123-156, :232-256,
:312-359) — with one 16-byte status read per attempt. The scale search
(bisection, or four probes per round from 1,500 islands, :405-468) and the
coarse-to-fine schedule (:491-532) drive the attempts from the host; without
a time budget the result is the reference's, placements and UVs bit for bit
(tests/golden/golden_pack.npz). The final UVs are computed on the device
from the placements (:537-549).

The maximal-contact placement (:169-220, :308-342) is not built: the
reference enables it for no chart (CONTACT_MAX_CHARTS = 0).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from .. import _lib
from ..device import require_cuda

ANGLES = (0.0,)
PROBES = 1
MANY_CHARTS = 1500
CONTACT_MIN_FRACTION = 0.004
CONTACT_MAX_CHARTS = 0
ORDERINGS = ("area", "bbox", "height")


# ------------------------------------------------------------------ orientation (host)
def min_area_rect_angle(U):
    """The convex-hull edge angle, modulo 90 degrees and rounded to 9 digits,
    whose rotation gives the smallest bounding rectangle (pack.py:19-37)."""
    from scipy.spatial import ConvexHull
    if len(U) < 3:
        return 0.0
    try:
        hull = U[ConvexHull(U).vertices]
    except Exception:  # noqa: BLE001 - degenerate point set: no rotation, as the reference
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


def orient(U, upright=None):
    """A chart turned to its minimum-area rectangle, landscape, minimum 0
    (pack.py:40-48)."""
    a = min_area_rect_angle(U)
    c, s = np.cos(-a), np.sin(-a)
    V = U @ np.array([[c, -s], [s, c]]).T
    ext = V.max(0) - V.min(0)
    if ext[1] > ext[0]:
        V = V[:, ::-1] * np.array([1, -1])
    return V - V.min(0)


def _rotated(U, a):
    """pack.py:365-370."""
    if a == 0.0:
        return U
    c, s_ = np.cos(a), np.sin(a)
    V = U @ np.array([[c, -s_], [s_, c]]).T
    return V - V.min(0)


def _uv_area(U, T):
    """pack.py:570-572."""
    a, b, c = U[T[:, 0]], U[T[:, 1]], U[T[:, 2]]
    return float(np.abs(0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1])
                               - (c[:, 0] - a[:, 0]) * (b[:, 1] - a[:, 1]))).sum())


def mask_shape(vmax, scale, pad):
    """(h, w) of a chart mask (pack.py:84-86) from the chart's largest x and
    y: fl(fl(u s) + pad) grows with u, so the largest scaled coordinate is
    the scaled largest one. Vectorised over rows of vmax."""
    vmax = np.asarray(vmax, np.float64)
    w = np.ceil(vmax[..., 0] * scale + pad + pad).astype(np.int64) + 1
    h = np.ceil(vmax[..., 1] * scale + pad + pad).astype(np.int64) + 1
    if np.ndim(w) == 0:
        return int(h), int(w)
    return h, w


# ------------------------------------------------------------------ device attempts
class _AttemptDesc(C.Structure):
    """Mirror of ``uva_pack_attempt``."""
    _fields_ = [("nsrc", C.c_int32), ("nc", C.c_int32), ("nk", C.c_int32), ("G", C.c_int32), ("pad", C.c_int32),
                ("reserved", C.c_int32), ("ntri", C.c_int64), ("ncells", C.c_int64), ("nrows", C.c_int64),
                ("run_cap", C.c_int64)] + [(n, C.c_void_p) for n in (
                    "V", "vofs", "T", "tofs", "scale", "hw", "mofs", "var_src", "var_turn", "var_row", "order",
                    "mask", "row_need", "run_ofs", "run_a", "run_b", "var_area", "var_key", "R", "rowmax",
                    "placement", "status", "occupied", "scratch")] + [("scratch_bytes", C.c_int64)]


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _upload(dev, *arrays):
    """Several small host arrays in one host-to-device copy; device views
    in the arrays' own dtypes."""
    offs, total = [], 0
    for a in arrays:
        total = (total + 15) & ~15
        offs.append(total)
        total += a.nbytes
    buf = np.zeros(max(total, 16), np.uint8)
    for a, o in zip(arrays, offs):
        buf[o:o + a.nbytes] = np.ascontiguousarray(a).view(np.uint8).ravel()
    d = torch.from_numpy(buf).to(dev, non_blocking=False)
    out = []
    for a, o in zip(arrays, offs):
        dt = {np.dtype(np.float64): torch.float64, np.dtype(np.int64): torch.int64,
              np.dtype(np.int32): torch.int32}[a.dtype]
        out.append(d[o:o + a.nbytes].view(dt))
    return out


class Attempt:
    """One successful packing attempt: the scale, the device placement
    (variant, x, y per chart) and the page occupancy."""

    def __init__(self, s, G, pad, hw, placement, occupied, nturns, nangles):
        self.s, self.G, self.pad = s, G, pad
        self.hw, self.placement_dev, self.occupied = hw, placement, occupied
        self.nturns, self.nangles = nturns, nangles

    @property
    def placement(self):
        """[(k, x, y)] per chart (k = angle index * turns + turn)."""
        p = self.placement_dev.view(-1, 3).cpu().numpy()
        return [tuple(int(v) for v in row) for row in p]

    @property
    def occupancy(self):
        """Occupied fraction of the planning page (occ.mean(), pack.py:551)."""
        return float(self.occupied / (self.G * self.G))


class Packer:
    """The oriented charts of one pack() call on the device, at every
    pre-rotation angle (mask source c * len(angles) + a), and packing
    attempts over them."""

    def __init__(self, Us, Ts, dens, angles=(0.0,), dev=None):
        self.dev = dev if dev is not None else require_cuda()
        self.nc = len(Us)
        self.angles = tuple(float(a) for a in angles)
        self.nA = len(self.angles)
        self.dens = np.asarray(dens, np.float64)
        src_U = [_rotated(U, a) for U in Us for a in self.angles]
        src_T = [T for T in Ts for _ in self.angles]
        nv = np.array([len(U) for U in src_U], np.int64)
        nt = np.array([len(T) for T in src_T], np.int64)
        self.vofs_h = np.concatenate([[0], np.cumsum(nv)]).astype(np.int64)
        self.tofs_h = np.concatenate([[0], np.cumsum(nt)]).astype(np.int64)
        self.vmax = np.array([U.max(0) if len(U) else (0.0, 0.0) for U in src_U], np.float64).reshape(-1, 2)
        self.ntri = int(self.tofs_h[-1])
        V = np.ascontiguousarray(np.concatenate(src_U) if src_U else np.zeros((0, 2)), np.float64)
        T = np.ascontiguousarray(np.concatenate(src_T) if src_T else np.zeros((0, 3)), np.int64)
        if T.size and (T.min() < 0 or (T.max(1) >= np.repeat(nv, nt)).any()):
            raise IndexError("pack: a triangle index is outside its chart")
        cn = np.array([len(U) for U in Us], np.int64)
        self.cofs_h = np.concatenate([[0], np.cumsum(cn)]).astype(np.int64)
        self.V = torch.from_numpy(V).to(self.dev)
        self.T = torch.from_numpy(T.astype(np.int32)).to(self.dev)
        self.vofs, self.tofs, self.cofs, self.dens_d = _upload(self.dev, self.vofs_h, self.tofs_h, self.cofs_h,
                                                               self.dens)
        self.attempts = 0
        self.seconds = 0.0

    # ---- sizes of one attempt (host, from the vertex maxima alone)
    def _layout(self, s, pad, rot_set):
        nr = len(rot_set)
        scale = np.repeat(s * self.dens, self.nA)
        h, w = mask_shape(self.vmax, scale, pad)
        h, w = np.atleast_1d(h), np.atleast_1d(w)
        tiny = h * w < 400
        nk = self.nA * nr
        turns = np.tile(np.array(rot_set, np.int32), self.nc * self.nA)
        src = np.repeat(np.arange(self.nc * self.nA, dtype=np.int32), nr)
        ang = np.tile(np.repeat(np.array(self.angles), nr), self.nc)
        none = tiny[src] & ((turns >= 2) | (ang != 0.0)) if len(src) else np.zeros(0, bool)
        var_src = np.where(none, -1, src).astype(np.int32)
        vh = np.where(none, 0, np.where(turns & 1, w[src], h[src])) if len(src) else np.zeros(0, np.int64)
        vw = np.where(none, 0, np.where(turns & 1, h[src], w[src])) if len(src) else np.zeros(0, np.int64)
        var_row = np.concatenate([[0], np.cumsum(vh)]).astype(np.int64)
        mofs = np.concatenate([[0], np.cumsum(h * w)]).astype(np.int64)
        hw = np.stack([h, w], 1).astype(np.int32).ravel()
        run_cap = int((vh * ((vw + 1) // 2)).sum())
        return dict(nk=nk, scale=scale, h=h, w=w, hw=hw, mofs=mofs, var_src=var_src, var_turn=turns,
                    var_row=var_row, run_cap=run_cap)

    def _masks(self, G, pad, rot_set, s, extra=()):
        """Launch the masks and runs of every variant at texel scale s; the
        descriptor, the layout, the device arrays and the uploads in extra."""
        L = _lib.lib()
        lay = self._layout(s, pad, rot_set)
        nk, nc, dev = lay["nk"], self.nc, self.dev
        nvar = nc * nk
        ncells, nrows = int(lay["mofs"][-1]), int(lay["var_row"][-1])
        scale, hw, mofs, var_src, var_turn, var_row, *rest = _upload(
            dev, lay["scale"], lay["hw"], lay["mofs"], lay["var_src"], lay["var_turn"], lay["var_row"], *extra)
        i32 = dict(dtype=torch.int32, device=dev)
        i64 = dict(dtype=torch.int64, device=dev)
        A = dict(scale=scale, hw=hw, mofs=mofs, var_src=var_src, var_turn=var_turn, var_row=var_row,
                 mask=torch.empty(max(ncells, 1), dtype=torch.uint8, device=dev),
                 row_need=torch.empty(max(nrows, 1), **i32), run_ofs=torch.empty(nrows + 1, **i32),
                 run_a=torch.empty(max(lay["run_cap"], 1), **i32), run_b=torch.empty(max(lay["run_cap"], 1), **i32),
                 var_area=torch.empty(max(nvar, 1), **i64), var_key=torch.empty(max(nvar, 1), **i64),
                 R=torch.empty(G * G, **i32), rowmax=torch.empty(G, **i32),
                 placement=torch.empty(max(3 * nc, 3), **i32), status=torch.empty(4, **i32),
                 occupied=torch.empty(1, **i64))
        nb = C.c_int64()
        _lib.check(L.uva_pack_scratch_bytes(self.ntri, ncells, nrows, nk, G, C.byref(nb)), "uva_pack_scratch_bytes")
        A["scratch"] = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
        d = _AttemptDesc(nsrc=nc * self.nA, nc=nc, nk=nk, G=G, pad=pad, ntri=self.ntri, ncells=ncells, nrows=nrows,
                         run_cap=lay["run_cap"], V=_ptr(self.V), vofs=_ptr(self.vofs), T=_ptr(self.T),
                         tofs=_ptr(self.tofs), scratch_bytes=A["scratch"].numel(),
                         **{k: _ptr(v) for k, v in A.items()})
        _lib.check(L.uva_pack_masks(C.byref(d), _stream(dev)), "uva_pack_masks")
        return d, lay, A, rest

    def masks(self, s, pad, rot_set=(0,)):
        """Per chart the list of variant masks (numpy, None for a tiny
        island's dropped turns) at texel scale s (pack.py:373-388)."""
        d, lay, A, _ = self._masks(1, pad, list(rot_set), s)
        mask = A["mask"].cpu().numpy()
        st = A["status"].cpu().numpy()
        if st[2]:
            raise RuntimeError("uva_pack_masks: run table capacity exceeded")
        out = []
        for c in range(self.nc):
            ms = []
            for a in range(self.nA):
                src = c * self.nA + a
                m0 = mask[lay["mofs"][src]:lay["mofs"][src + 1]].reshape(lay["h"][src], lay["w"][src])
                for j, r in enumerate(rot_set):
                    ms.append(None if lay["var_src"][(c * self.nA + a) * len(rot_set) + j] < 0
                              else np.ascontiguousarray(np.rot90(m0, r)))
            out.append(ms)
        return out

    def _prepare(self, G, pad, rot_set, s, ordering):
        """Masks and runs at texel scale s and the placing order; the
        descriptor (order set) and what it points to."""
        if ordering not in ORDERINGS:
            raise ValueError(f"unknown ordering {ordering!r}")
        extra = ()
        if ordering != "area":
            lay = self._layout(s, pad, rot_set)
            h0, w0 = lay["h"][::self.nA], lay["w"][::self.nA]
            key = h0 * w0 if ordering == "bbox" else np.minimum(h0, w0)
            extra = (np.argsort(-key, kind="stable").astype(np.int64),)
        d, lay, A, rest = self._masks(G, pad, rot_set, s, extra)
        nc, nk = self.nc, lay["nk"]
        if ordering == "area":    # decreasing set cells of angle 0, turn 0, stable
            order = torch.argsort(-A["var_area"][:nc * nk].view(nc, nk)[:, 0], stable=True) if nc else A["var_area"][:0]
        else:
            order = rest[0]
        A["order"] = order.contiguous()
        d.order = _ptr(A["order"])
        return d, lay, A

    def _result(self, s, G, pad, rot_set, lay, A, st):
        if st[2]:
            raise RuntimeError("uva_pack_masks: run table capacity exceeded")
        if st[0] & 2:
            raise RuntimeError("uva_pack_place: grid barrier timed out")
        if st[0] & 1:
            return None
        return Attempt(s, G, pad, lay["hw"].reshape(-1, 2), A["placement"], int(A["occupied"].item()),
                       len(rot_set), self.nA)

    def attempt(self, G, pad, rot_set, s, ordering="area", blocks_per_sm=0):
        """Masks at texel scale s, then the first fit of every chart on a
        G x G page: an Attempt, or None when a chart fits nowhere
        (pack.py:398-402)."""
        t0 = time.perf_counter()
        d, lay, A = self._prepare(G, pad, rot_set, s, ordering)
        _lib.check(_lib.lib().uva_pack_place(C.byref(d), int(blocks_per_sm), _stream(self.dev)), "uva_pack_place")
        st = A["status"].cpu().numpy()
        self.attempts += 1
        self.seconds += time.perf_counter() - t0
        return self._result(s, G, pad, rot_set, lay, A, st)

    def attempts_at(self, G, pad, rot_set, scales, ordering="area", blocks_per_sm=0):
        """Up to four attempts at different scales placed in one launch (the
        probes of one k-ary search round): a list of Attempt or None."""
        t0 = time.perf_counter()
        prep = [self._prepare(G, pad, rot_set, s, ordering) for s in scales]
        descs = (C.c_void_p * len(prep))(*[C.cast(C.pointer(d), C.c_void_p) for d, _, _ in prep])
        _lib.check(_lib.lib().uva_pack_place_pages(descs, len(prep), int(blocks_per_sm), _stream(self.dev)),
                   "uva_pack_place_pages")
        sts = torch.stack([A["status"] for _, _, A in prep]).cpu().numpy()
        self.attempts += len(prep)
        self.seconds += time.perf_counter() - t0
        return [self._result(s, G, pad, rot_set, lay, A, st) for s, (_, lay, A), st in zip(scales, prep, sts)]

    def uvs(self, att):
        """Per chart the UVs in [0, 1] of a successful attempt
        (pack.py:537-549)."""
        L = _lib.lib()
        nv = int(self.cofs_h[-1])
        out = torch.empty(max(nv, 1), 2, dtype=torch.float64, device=self.dev)
        hw = _upload(self.dev, att.hw.astype(np.int32).ravel())[0]
        d = _AttemptDesc(nsrc=self.nc * self.nA, nc=self.nc, nk=self.nA * att.nturns, G=att.G, pad=att.pad,
                         V=_ptr(self.V), vofs=_ptr(self.vofs), hw=_ptr(hw), placement=_ptr(att.placement_dev))
        _lib.check(L.uva_pack_uv(C.byref(d), self.nA, att.nturns, _ptr(self.cofs), nv, C.c_double(att.s),
                                 _ptr(self.dens_d), _ptr(out), _stream(self.dev)), "uva_pack_uv")
        uv = out[:nv].cpu().numpy()
        return [uv[self.cofs_h[i]:self.cofs_h[i + 1]] for i in range(self.nc)]


def chart_mask(U, T, scale, pad):
    """The (h, w) uint8 mask of an oriented chart (minimum 0) at `scale`
    texels per unit with a `pad`-texel border, dilated by `pad`
    (pack.py:82-92), rasterised on the device."""
    P = Packer([np.asarray(U, np.float64)], [np.ascontiguousarray(T, np.int64)], [1.0])
    return P.masks(float(scale), int(pad))[0][0]


# ------------------------------------------------------------------ scale search (host)
def _search(attempt_fn, n, s, iters, tol=0.004, lo=0.0, hi=None, best=None, deadline=None):
    """pack.py:409-415: four probes per round from MANY_CHARTS islands (or
    PROBES > 1), else bisection. attempt_fn(scale) -> Attempt or None."""
    if PROBES > 1 or n >= MANY_CHARTS:
        return _search_kary(attempt_fn, s, iters, tol, lo, hi, best, deadline)
    return _search_bisect(attempt_fn, s, iters, tol, lo, hi, best, deadline)


def _search_kary(attempt_fn, s, iters, tol, lo, hi, best, deadline):
    """pack.py:418-445: the bracket shrinks about five times per round of
    four probes; the probes of a round share one placement launch (only
    which of them fit decides the next round)."""
    k = max(PROBES, 4)
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
        many = getattr(attempt_fn, "many", None)
        res = many([float(sc) for sc in cand]) if many else [attempt_fn(float(sc)) for sc in cand]
        for sc, r in zip(cand, res):
            if r is not None and sc > lo:
                best, lo = r, float(sc)
        fails = [float(sc) for sc, r in zip(cand, res) if r is None and sc > lo]
        if fails:
            hi = min(fails) if hi is None else min(hi, min(fails))
    return best, lo, hi


def _search_bisect(attempt_fn, s, iters, tol, lo, hi, best, deadline):
    """pack.py:448-468: grow by 1.2 until an attempt fails, shrink by 0.8
    until one fits, then bisect the bracket."""
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


def pack(charts, atlas=4096, padding=4, grid=None, rotations=4, density=None, iters=10, log=None,
         time_budget=None, orderings=("area", "bbox", "height"), angles=(0.0,), fine_attempts=8):
    """charts: list of (U, T) in 3D units; density: per-chart linear texel
    multipliers. Returns the per-chart UVs in [0, 1] and an info dict
    (pack.py:471-554). From a 1024-texel planning grid the scale search runs
    coarse-to-fine: every ordering on the half grid, then a short climb and
    bisection on the full grid."""
    global ANGLES
    t0 = time.perf_counter()
    ANGLES = tuple(float(a) for a in angles)
    deadline = None if not time_budget else t0 + float(time_budget)
    grid = grid or min(atlas, 2048)
    pad = int(np.ceil(padding * grid / atlas))
    n = len(charts)
    dens = np.ones(n) if density is None else np.asarray(density, float)
    Us = [orient(U) for U, _ in charts]
    Ts = [np.ascontiguousarray(T, np.int64) for _, T in charts]
    area = np.array([_uv_area(U, T) * d * d for U, T, d in zip(Us, Ts, dens)])
    tot = max(area.sum(), 1e-30)
    rot_set = [0, 1, 2, 3][:max(1, rotations)]
    P = Packer(Us, Ts, dens, ANGLES)

    def at(G, p, o):
        fn = lambda sc: P.attempt(G, p, rot_set, sc, o)  # noqa: E731
        fn.many = lambda scs: P.attempts_at(G, p, rot_set, scs, o)
        return fn

    best = None
    if grid >= 1024:
        g2 = grid // 2
        pad2 = max(1, int(np.ceil(padding * g2 / atlas)))
        b2, ordering = None, orderings[0]
        for o in orderings:    # multi-start: the ordering reaching the largest coarse scale wins
            if deadline is not None and b2 is not None and time.perf_counter() > t0 + 0.4 * float(time_budget):
                break
            s0 = b2.s if b2 is not None else np.sqrt(0.62 * g2 * g2 / tot)
            bo, _, _ = _search(at(g2, pad2, o), n, s0, iters, tol=0.01,
                               deadline=None if deadline is None else t0 + 0.6 * float(time_budget))
            if bo is not None and (b2 is None or bo.s > b2.s):
                b2, ordering = bo, o
        if b2 is not None:
            s0 = b2.s * grid / g2 * 0.98    # just under the coarse estimate
            r, used = None, 0
            for _ in range(4):
                r = P.attempt(grid, pad, rot_set, s0, ordering)
                used += 1
                if r is not None:
                    break
                s0 *= 0.96
            if r is not None:
                # the coarse masks are conservative: climb while the full grid still fits, then bisect
                lo_, hi_ = s0, s0 * 1.06
                for _ in range(8):
                    if (deadline is not None and time.perf_counter() > deadline) or used >= fine_attempts:
                        break
                    used += 1
                    r2 = P.attempt(grid, pad, rot_set, hi_, ordering)
                    if r2 is None:
                        break
                    r, lo_, hi_ = r2, hi_, hi_ * 1.06
                best = r
                if fine_attempts - used > 0:
                    best, _, _ = _search(at(grid, pad, ordering), n, 0.5 * (lo_ + hi_), min(3, fine_attempts - used),
                                         tol=0.006, lo=lo_, hi=hi_, best=r, deadline=deadline)
    if best is None:
        best, _, _ = _search(at(grid, pad, "area"), n, np.sqrt(0.62 * grid * grid / tot), iters)
    if best is None:
        raise RuntimeError("packing failed: charts do not fit one page even at small scale")
    uvs = P.uvs(best)
    s = best.s
    info = {"texel_scale_grid": s, "texels_per_unit_atlas": s * atlas / grid, "grid": grid, "grid_padding": pad,
            "plan_occupancy": best.occupancy, "seconds": time.perf_counter() - t0,
            "attempts": P.attempts, "attempt_seconds": P.seconds}
    if log:
        log(f"pack: {n} charts grid {grid} pad {pad} scale {s:.4g} occ(dilated) {best.occupancy:.3f} "
            f"{info['seconds']:.1f}s")
    return uvs, info
