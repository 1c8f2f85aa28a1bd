"""Device-resident batch of islands and the calls into the CUDA library.

A ``DeviceBatch`` concatenates many charts block-diagonally, builds the
topology plan on the host cores (C++, parallel over islands), uploads it once,
and keeps every per-island array in HBM: frames, weights, the sliced-ELL
Laplacian, UVs and solver scratch. All solver calls run on one CUDA stream and
never synchronise the host.

Memory: about 80 bytes per triangle plus about 180 bytes per vertex
(UVs, solver vectors, sliced-ELL slots) and 20 bytes per squared coarse
aggregate, so a 180 GB B200 holds batches of several hundred million
triangles.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import threading

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr

# ARAP solves each global step to 2e-7 relative residual per column: at 1e-6
# the UVs after 20 outer iterations drift up to 3e-5 (relative to the chart's
# UV extent) from exact solves on 2,000 uneven islands; at 2e-7 they stay
# below 4e-6, for about 13 % more CG iterations. Inner FP32 solves aim at a
# 1e-5 reduction (or the final tolerance): fewer FP64 restarts than 1e-3.
# LSCM solves to 1e-8: on the same islands (12 size-stratified ones against
# the FP64 oracle) the LSCM UVs stay within 4.5e-7 of exact solves and the
# UVs after 20 ARAP iterations within 2e-6, for 5 % less LSCM time than
# 1e-9; at 1e-7 the LSCM error grows to 6e-6, at 1e-6 to 9e-5.
DEFAULTS = {
    "arap": {"tol": 2e-7, "inner_eta": 1e-5, "max_inner": 4000, "max_refine": 12},
    "lscm": {"tol": 1e-8, "inner_eta": 1e-3, "max_inner": 20000, "max_refine": 16},
}


def require_cuda(dev=None):
    """The product path has no CPU fallback: fail loudly without a CUDA device."""
    if not torch.cuda.is_available():
        raise RuntimeError("ultimate_uv_artist_b200 needs a CUDA device (sm_100a); none is available")
    d = torch.device(dev) if dev is not None else torch.device("cuda", torch.cuda.current_device())
    if d.type != "cuda":
        raise RuntimeError(f"ultimate_uv_artist_b200 runs on CUDA devices only, got {d}")
    return d


def host_empty(shape, dtype):
    """numpy array in page-locked host memory when CUDA is present (torch's
    caching host allocator: reused across batches), so uploads are plain
    asynchronous DMA; ordinary memory otherwise."""
    if torch.cuda.is_available():
        n = int(np.prod(shape)) if np.ndim(shape) else int(shape)
        t = torch.empty(max(n, 1), dtype=_TORCH_OF[np.dtype(dtype)], pin_memory=True)
        return t.numpy()[:n].reshape(shape)
    return np.empty(shape, dtype)


_TORCH_OF = {np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64, np.dtype(np.float32): torch.float32,
             np.dtype(np.float64): torch.float64, np.dtype(np.uint8): torch.uint8}
_NUMPY_OF = {v: k for k, v in _TORCH_OF.items()}


def to_host(t):
    """A device tensor's contents as a numpy array in page-locked memory
    (torch's caching host allocator, so repeated calls reuse it instead of
    page-faulting fresh pageable memory): one asynchronous copy on the
    current stream, then a wait for it."""
    if t.dtype not in _NUMPY_OF:
        return t.cpu().numpy()
    out = host_empty(tuple(t.shape), _NUMPY_OF[t.dtype])
    if t.numel():
        torch.from_numpy(out).copy_(t, non_blocking=True)
        torch.cuda.current_stream(t.device).synchronize()
    return out


class Plan:
    """Host topology plan (wraps uva_plan_create / uva_plan_export)."""

    # the arrays uva_plan_export writes, island by island
    EXPORTED = ("tri4", "tri_edge", "sofs", "slice_ptr", "slot_col", "slot_edge", "slot_c", "vt_ptr", "vt", "vflags",
                "bofs", "bverts")

    def __init__(self, T_local, vofs, tofs, nthreads=0, chart_tris=None, device=None, stream=None, chunks=4):
        """T_local: concatenated island-local triangles; or None with
        ``chart_tris`` = (pointer array, dtype code array) of per-chart
        triangle arrays (uva_plan_create_charts: no concatenation).

        With ``device``, the plan's arrays are also copied to that device
        (``dev_arrays``): the export runs in ``chunks`` island ranges and the
        copies of each finished range run on ``stream`` while the next range
        is exported."""
        L = _lib.lib()
        vofs = np.ascontiguousarray(vofs, np.int64)
        tofs = np.ascontiguousarray(tofs, np.int64)
        nc = len(vofs) - 1
        h = C.c_void_p()
        if chart_tris is not None:
            tp, tdt = chart_tris
            check(L.uva_plan_create_charts(ptr(tp), ptr(tdt), ptr(vofs), ptr(tofs), nc, int(nthreads), C.byref(h)),
                  "uva_plan_create")
        else:
            T_local = np.ascontiguousarray(T_local, np.int64).reshape(-1, 3)
            check(L.uva_plan_create(ptr(T_local), ptr(vofs), ptr(tofs), nc, int(nthreads), C.byref(h)),
                  "uva_plan_create")
        self.dev_arrays = None
        try:
            sz = np.zeros(_lib.PLAN_NSIZES, np.int64)
            check(L.uva_plan_sizes(h, ptr(sz)), "uva_plan_sizes")
            self.nc, self.n, self.t, self.E = int(sz[0]), int(sz[1]), int(sz[2]), int(sz[3])
            self.nslices, self.nslots, self.nbverts, self.maxrows = int(sz[4]), int(sz[5]), int(sz[6]), int(sz[7])
            self.ncoarse = int(sz[8])
            self.tri4 = host_empty((self.t, 4), np.int32)
            self.tri_edge = host_empty((self.t, 3), np.int32)
            self.sofs = host_empty(nc + 1, np.int32)
            self.slice_ptr = host_empty(self.nslices + 1, np.int32)
            self.slot_col = host_empty(self.nslots, np.int32)
            self.slot_edge = host_empty(self.nslots, np.int32)
            self.slot_c = host_empty(self.nslots, np.float32)
            self.vt_ptr = host_empty(self.n + 1, np.int32)
            self.vt = host_empty(3 * self.t, np.int32)
            self.vflags = host_empty(self.n, np.uint8)
            self.bofs = host_empty(nc + 1, np.int32)
            self.bverts = host_empty(max(self.nbverts, 1), np.int32)
            args = [ptr(getattr(self, k)) for k in self.EXPORTED]
            if device is None or nc == 0:
                check(L.uva_plan_export(h, *args), "uva_plan_export")
            else:
                self._export_to_device(L, h, args, vofs, tofs, device, stream, max(int(chunks), 1))
            self.row_vert = host_empty(max(self.n, 1), np.int32)
            self.vert_row = host_empty(max(self.n, 1), np.int32)
            self.agg_rows = host_empty(max(nc, 1), np.int32)
            self.cofs = host_empty(nc + 1, np.int32)
            check(L.uva_plan_export_rows(h, ptr(self.row_vert), ptr(self.vert_row), ptr(self.agg_rows), ptr(self.cofs)),
                  "uva_plan_export_rows")
        finally:
            # freeing the plan's per-island buffers takes a few ms: off the
            # caller's path (ctypes releases the GIL during the call)
            threading.Thread(target=L.uva_plan_destroy, args=(h,), daemon=True).start()
        self.vofs = vofs.astype(np.int32)
        self.tofs = tofs.astype(np.int32)
        # island work order: grouped by size class (whole CTA with global or
        # shared-memory vectors, 256-thread sub-team, warp), largest first
        self.set_classes(_lib.CLASS_MID, _lib.CLASS_SMALL)

    def _export_to_device(self, L, h, args, vofs, tofs, device, stream, chunks):
        """Export island ranges of about equal triangle counts and copy each
        finished range (page-locked, asynchronous) to its device arrays."""
        nc = self.nc
        off = np.zeros(3 * (nc + 1), np.int64)
        check(L.uva_plan_island_offsets(h, ptr(off)), "uva_plan_island_offsets")
        so, sl, bo = off[:nc + 1], off[nc + 1:2 * (nc + 1)], off[2 * (nc + 1):]
        vr, tr = vofs - int(vofs[0]), tofs - int(tofs[0])
        # first element of island i in every exported array
        starts = {"tri4": 4 * tr, "tri_edge": 3 * tr, "sofs": np.arange(nc + 1), "slice_ptr": so, "slot_col": sl,
                  "slot_edge": sl, "slot_c": sl, "vt_ptr": vr, "vt": 3 * tr, "vflags": vr, "bofs": np.arange(nc + 1),
                  "bverts": bo}
        closing = {"sofs", "slice_ptr", "vt_ptr", "bofs"}   # one entry past the last island
        dev = {k: torch.empty(max(getattr(self, k).size, 1), dtype=_TORCH_OF[getattr(self, k).dtype], device=device)
               for k in self.EXPORTED}
        cuts = np.searchsorted(tr, np.linspace(0, tr[-1], chunks + 1)[1:-1])
        bounds = [0] + sorted(set(int(c) for c in cuts if 0 < c < nc)) + [nc]
        ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
        for i0, i1 in zip(bounds[:-1], bounds[1:]):
            check(L.uva_plan_export_range(h, i0, i1, *args), "uva_plan_export_range")
            with ctx:
                for k in self.EXPORTED:
                    a, b = int(starts[k][i0]), int(starts[k][i1]) + (1 if (k in closing and i1 == nc) else 0)
                    if b > a:
                        dev[k][a:b].copy_(torch.from_numpy(getattr(self, k).reshape(-1)[a:b]), non_blocking=True)
        self.dev_arrays = {k: v.view(getattr(self, k).shape) if getattr(self, k).size else v for k, v in dev.items()}

    def set_classes(self, mid, small):
        """Island work order for team thresholds ``mid`` (whole CTA above) and
        ``small`` (sub-team above, warp at or below); islands above
        CLASS_BIG vertices keep global-memory vectors. The kernels' team
        capacities bound them: mid <= CLASS_MID, small <= CLASS_SMALL."""
        mid = int(min(mid, _lib.CLASS_MID))
        small = int(min(small, _lib.CLASS_SMALL, mid))
        nv = np.diff(self.vofs.astype(np.int64))
        cls = np.where(nv > _lib.CLASS_BIG, 0, np.where(nv > mid, 1, np.where(nv > small, 2, 3)))
        self.order = np.lexsort((-nv, cls)).astype(np.int32)
        self.class_ofs = np.searchsorted(cls[self.order], np.arange(5)).astype(np.int32)
        self.classes = (mid, small)


def coarse_sizes(nv):
    """Rows per coarse aggregate, aggregates and coarse-block offsets of
    islands with ``nv`` vertices (plan.cpp's rule: no coarse level up to 256
    vertices, else the smallest multiple of 64 rows giving at most 256
    aggregates), and the 32-row slice offsets."""
    nv = np.asarray(nv, np.int64)
    agg = np.where(nv > 256, 64 * np.maximum(1, -(-nv // (256 * 64))), 0).astype(np.int64)
    ncoarse = np.where(agg > 0, -(-nv // np.maximum(agg, 1)), 0)
    cofs = np.zeros(len(nv) + 1, np.int64)
    np.cumsum(ncoarse * ncoarse, out=cofs[1:])
    sofs = np.zeros(len(nv) + 1, np.int64)
    np.cumsum(-(-nv // 32), out=sofs[1:])
    return agg, ncoarse, cofs, sofs


class DevicePlan:
    """The topology plan built on the device (uva_dplan_build /
    uva_dplan_slots): the arrays of Plan, element for element, from the
    charts' island-local triangles. The host concatenates the triangles as
    int32 (page-locked, in parallel), uploads them with the offsets and the
    size-only quantities (aggregate rows, slice and coarse offsets), and
    reads back four sizes. Host copies of the arrays are made on first
    access (``plan.slot_edge`` etc.), for the bench's statistics."""

    EXPORTED = Plan.EXPORTED
    on_device = True

    def __init__(self, chart_tris, vofs, tofs, device, stream=None, finish=True):
        """Launches the build on ``stream``; with ``finish`` False the caller
        runs host work of its own and then calls finish() (which waits for
        the build's sizes and launches the slot pass)."""
        L = _lib.lib()
        d = require_cuda(device)
        vofs = np.ascontiguousarray(vofs, np.int64)
        tofs = np.ascontiguousarray(tofs, np.int64)
        nc = len(vofs) - 1
        if nc and (vofs[0] != 0 or tofs[0] != 0 or (np.diff(vofs) < 0).any() or (np.diff(tofs) < 0).any()):
            raise ValueError("DevicePlan: offsets must start at 0 and not decrease")
        self.nc, self.n, self.t = nc, int(vofs[-1]), int(tofs[-1])
        nv = np.diff(vofs)
        if self.n > (1 << 30) or 3 * self.t > (1 << 30):
            raise ValueError("uva_plan_create: batch too large for 32-bit indices")
        if nc and int(nv.max()) >= (1 << 24):
            raise ValueError("uva_plan_create: island above 16M vertices")
        agg, ncoarse, cofs, sofs = coarse_sizes(nv)
        self.nslices = int(sofs[-1])
        self.ncoarse = int(cofs[-1])
        self.maxrows = int(nv.max()) if nc else 0
        self.vofs = vofs.astype(np.int32)
        self.tofs = tofs.astype(np.int32)
        self.h2d_bytes = 0
        tp, tdt = chart_tris[0], chart_tris[1]
        T32 = host_empty((max(self.t, 1), 3), np.int32)
        if nc:
            check(L.uva_concat_tris32(nc, ptr(tp), ptr(tdt), ptr(tofs), ptr(T32), 0), "uva_concat_tris32")
        ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
        with ctx:
            def up(a):
                t = torch.from_numpy(np.ascontiguousarray(a))
                self.h2d_bytes += t.numel() * t.element_size()
                return t.to(d, non_blocking=t.is_pinned())
            i32 = torch.int32
            vd, td = up(self.vofs), up(self.tofs)
            Td = up(T32)
            self.agg_rows = up(agg.astype(np.int32) if nc else np.zeros(1, np.int32))
            self.cofs = up(cofs.astype(np.int32))
            sofs_d = up(sofs.astype(np.int32))
            n1, t1 = max(self.n, 1), max(self.t, 1)
            dev = {"tri4": torch.empty((t1, 4), dtype=i32, device=d), "tri_edge": torch.empty((t1, 3), dtype=i32, device=d),
                   "sofs": sofs_d, "slice_ptr": torch.empty(self.nslices + 1, dtype=i32, device=d),
                   "vt_ptr": torch.empty(self.n + 1, dtype=i32, device=d), "vt": torch.empty(3 * t1, dtype=i32, device=d),
                   "vflags": torch.empty(n1, dtype=torch.uint8, device=d), "bofs": torch.empty(nc + 1, dtype=i32, device=d),
                   "bverts": torch.empty(n1, dtype=i32, device=d)}
            self.row_vert = torch.empty(n1, dtype=i32, device=d)
            self.vert_row = torch.empty(n1, dtype=i32, device=d)
            sizes = torch.zeros(4, dtype=torch.int64, device=d)
            nb = C.c_int64()
            check(L.uva_dplan_scratch_bytes(self.n, self.t, self.nslices, C.byref(nb)), "uva_dplan_scratch_bytes")
            scratch = torch.empty(max(int(nb.value), 256), dtype=torch.uint8, device=d)
            D = _lib.DPlanDesc()
            D.nc, D.n, D.t, D.nslices = nc, self.n, self.t, self.nslices
            D.vofs, D.tofs, D.T, D.agg_rows, D.sofs = (vd.data_ptr(), td.data_ptr(), Td.data_ptr(),
                                                       self.agg_rows.data_ptr(), sofs_d.data_ptr())
            for k in ("tri4", "tri_edge", "slice_ptr", "vt_ptr", "vt", "vflags", "bofs", "bverts"):
                setattr(D, k, dev[k].data_ptr())
            D.row_vert, D.vert_row = self.row_vert.data_ptr(), self.vert_row.data_ptr()
            D.sizes, D.scratch, D.scratch_bytes = sizes.data_ptr(), scratch.data_ptr(), int(nb.value)
            s = stream if stream is not None else torch.cuda.current_stream(d)
            check(L.uva_dplan_build(C.byref(D), C.c_void_p(s.cuda_stream)), "uva_dplan_build")
        self._pending = (D, sizes, dev, s, d, Td, scratch, T32)
        self.dev_arrays = None
        if finish:
            self.finish()

    def finish(self):
        """Sizes of the build (waits for it), then the sliced-ELL slots."""
        if self._pending is None:
            return self
        L = _lib.lib()
        D, sizes, dev, s, d, Td, scratch, T32 = self._pending
        i32 = torch.int32
        sh = C.c_void_p(s.cuda_stream)
        with torch.cuda.stream(s):
            sz = sizes.cpu().numpy()     # waits for the build
            if sz[3] & 1:
                raise ValueError("uva_plan_create: triangle index outside its island")
            if sz[3] & 2:
                raise ValueError("uva_plan_create: an edge is used by more than 127 triangles in one direction")
            if sz[3] & 4:
                raise RuntimeError("uva_dplan_build: the row walk ran out of vertices")
            self.E, self.nslots, self.nbverts = int(sz[0]), int(sz[1]), int(sz[2])
            if self.nslots < 0:
                raise ValueError("uva_plan_create: plan too large for 32-bit offsets")
            for k, dt in (("slot_col", i32), ("slot_edge", i32), ("slot_c", torch.float32)):
                dev[k] = torch.empty(max(self.nslots, 1), dtype=dt, device=d)
            check(L.uva_dplan_slots(C.byref(D), dev["slot_col"].data_ptr(), dev["slot_edge"].data_ptr(),
                                    dev["slot_c"].data_ptr(), sh), "uva_dplan_slots")
            dev["bverts"] = dev["bverts"][:max(self.nbverts, 1)]
        self._keep = (Td, scratch, T32)   # in use until the stream passes the slot pass
        self._pending = None
        self.dev_arrays = dev
        self.set_classes(_lib.CLASS_MID, _lib.CLASS_SMALL)
        return self

    set_classes = Plan.set_classes

    def __getattr__(self, name):
        # host copies of the device arrays, made on first access
        if name in DevicePlan.EXPORTED:
            a = self.__dict__["dev_arrays"][name]
            sizes = {"bverts": self.nbverts, "slot_col": self.nslots, "slot_edge": self.nslots,
                     "slot_c": self.nslots, "vflags": self.n}
            out = a.cpu().numpy()
            if name in sizes:
                out = out[:sizes[name]]
            elif name in ("tri4", "tri_edge", "vt"):
                out = out[:self.t] if name != "vt" else out[:3 * self.t]
            self.__dict__[name] = out
            return out
        raise AttributeError(name)


_FLOAT_CODE = {np.dtype(np.float32): 0, np.dtype(np.float64): 1}
_INT_CODE = {np.dtype(np.int32): 0, np.dtype(np.int64): 1}


def _chart_array(a, width, codes, fallback):
    """(C-contiguous array of `width` columns, dtype code) without a copy
    when the dtype is one the concatenation reads directly."""
    a = np.asarray(a)
    if a.dtype not in codes:
        a = a.astype(fallback)
    a = np.ascontiguousarray(a).reshape(-1, width)
    return a, codes[a.dtype]


class ChartArrays:
    """Per-chart arrays of a batch, checked and C-contiguous (no copies when
    their dtypes are ones the host copies read), with dtype codes, pointer
    arrays and vertex / triangle offsets."""

    def __init__(self, charts, with_uv=True):
        nc = len(charts)
        self.nc = nc
        n1 = max(nc, 1)
        self.pdt = np.zeros(n1, np.int8)
        self.tdt = np.zeros(n1, np.int8)
        self.udt = np.full(n1, -1, np.int8)
        self.pp = np.zeros(n1, np.uintp)
        self.tp = np.zeros(n1, np.uintp)
        up = np.zeros(n1, np.uintp)
        nvs = np.zeros(n1, np.int64)
        nts = np.zeros(n1, np.int64)
        ok = np.zeros(n1, np.int8)
        ph = _lib.pyhost() if isinstance(charts, (list, tuple)) else None
        if ph is not None and nc:
            # one native pass: pointers, rows and codes of the arrays the host
            # copies read as they are; the other charts go through Python below
            ph.uva_py_charts(charts, 1 if with_uv else 0, ptr(self.pp), ptr(self.pdt), ptr(self.tp), ptr(self.tdt),
                             ptr(up), ptr(self.udt), ptr(nvs), ptr(nts), ptr(ok))
        self.Ps = [ch[0] for ch in charts]
        self.Ts = [ch[1] for ch in charts]
        self.Us = [(ch[2] if with_uv and len(ch) > 2 else None) for ch in charts]
        fc, ic = _FLOAT_CODE, _INT_CODE
        for i in np.flatnonzero(ok[:nc] == 0).tolist():
            ch = charts[i]
            a, self.pdt[i] = _chart_array(ch[0], 3, fc, np.float64)
            t, self.tdt[i] = _chart_array(ch[1], 3, ic, np.int64)
            self.Ps[i], self.Ts[i] = a, t
            nvs[i], nts[i] = a.shape[0], t.shape[0]
            self.pp[i], self.tp[i] = a.ctypes.data, t.ctypes.data
            u = None
            self.udt[i] = -1
            up[i] = 0
            if with_uv and len(ch) > 2 and ch[2] is not None:
                u, self.udt[i] = _chart_array(ch[2], 2, fc, np.float64)
                if len(u) != len(a):
                    raise ValueError(f"chart {i}: U has {len(u)} rows for {len(a)} vertices")
                up[i] = u.ctypes.data
            self.Us[i] = u
        self.up = up
        self.any_uv = bool(nc and (self.udt[:nc] >= 0).any())
        self.vofs = np.zeros(nc + 1, np.int64)
        self.tofs = np.zeros(nc + 1, np.int64)
        if nc:
            np.cumsum(nvs[:nc], out=self.vofs[1:])
            np.cumsum(nts[:nc], out=self.tofs[1:])

    @property
    def chart_tris(self):
        """(pointer array, dtype codes, arrays) of the triangles for the plans
        (the arrays stay referenced while a plan reads them)."""
        return self.tp, self.tdt, self.Ts

    def points(self, fp32=False):
        """(P, U): concatenated positions (page-locked; float32 when ``fp32``
        and every chart is float32 and none brings UVs, else FP64) and FP64
        UVs (None when no chart brings UVs), copied in parallel on the host."""
        nc, n = self.nc, int(self.vofs[-1])
        L = _lib.lib()
        U = host_empty((n, 2), np.float64) if self.any_uv else None
        if fp32 and nc and (self.pdt[:nc] == 0).all() and U is None:
            P = host_empty((n, 3), np.float32)
            check(L.uva_concat_rows32(nc, ptr(self.pp), ptr(self.vofs), 3, ptr(P), 0), "uva_concat_rows32")
            return P, None
        P = host_empty((n, 3), np.float64)
        if nc:
            up_ = self.up if self.any_uv else None
            check(L.uva_concat_charts(nc, ptr(self.pp), ptr(self.pdt), ptr(self.tp), ptr(self.tdt),
                                      ptr(up_) if self.any_uv else None, ptr(self.udt) if self.any_uv else None,
                                      ptr(self.vofs), ptr(self.tofs), ptr(P), None, ptr(U) if U is not None else None,
                                      0), "uva_concat_charts")
        return P, U


def concat_charts(charts, with_uv=True, with_t=True):
    """(P, T, U) per chart -> concatenated FP64 P, local int64 T, FP64 U, offsets
    (uva_concat_charts copies the charts in parallel; P and U in page-locked
    memory for the uploads). U is None when no chart brings UVs (nothing to
    upload: the device UVs start at zero). With ``with_t`` False the
    triangles are not copied: T is then (pointer array, dtype codes, arrays)
    of the per-chart arrays for Plan(chart_tris=...)."""
    ca = ChartArrays(charts, with_uv=with_uv)
    P, U = ca.points()
    if not with_t:
        return P, ca.chart_tris, U, ca.vofs, ca.tofs
    T = np.empty((int(ca.tofs[-1]), 3), np.int64)
    for t, a, b in zip(ca.Ts, ca.tofs[:-1], ca.tofs[1:]):
        T[a:b] = t
    return P, T, U, ca.vofs, ca.tofs


class DeviceBatch:
    """Islands resident on one CUDA device, ready for the uva_* kernels."""

    def __init__(self, P, T_local, vofs, tofs, U=None, semantics=_lib.SEM_BATCH, device=None, stream=None,
                 plan=None):
        self.dev = require_cuda(device)
        self.stream = stream
        self.semantics = int(semantics)
        plan = plan if plan is not None else Plan(T_local, vofs, tofs)
        self.plan = plan
        # a schedule tuned earlier for batches of this size signature (autotune)
        from . import autotune
        tuned = autotune.lookup(plan, self.dev)
        if tuned is not None:
            plan.set_classes(tuned["mid"], tuned["small"])
        # every copy and fill below runs on the batch stream, like its kernels
        with (torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()):
            self.nc, self.n, self.t = plan.nc, plan.n, plan.t
            d = self.dev

            self.h2d_bytes = 0   # bytes copied host -> device by this constructor

            def up(a, dtype=None):
                if isinstance(a, torch.Tensor):   # built on the device (DevicePlan)
                    t = a if a.numel() else torch.zeros(1, dtype=a.dtype, device=d)
                    return t.to(d) if dtype is None else t.to(d, dtype)
                t = torch.from_numpy(np.ascontiguousarray(a))
                if t.numel() == 0:
                    t = torch.zeros(1, dtype=t.dtype)
                self.h2d_bytes += t.numel() * t.element_size()
                # page-locked sources (the plan's arrays) copy asynchronously on
                # the current stream; the plan keeps them alive
                nb = t.is_pinned()
                return t.to(d, non_blocking=nb) if dtype is None else t.to(d, dtype, non_blocking=nb)

            # topology
            self.vofs = up(plan.vofs); self.tofs = up(plan.tofs); self.order = up(plan.order)
            pd = plan.dev_arrays if plan.dev_arrays is not None and plan.dev_arrays['tri4'].device == d else None
            built_on_device = getattr(plan, "on_device", False)
            if built_on_device:
                self.h2d_bytes += plan.h2d_bytes   # triangles and offsets; the plan's arrays were made there
            for k in Plan.EXPORTED:   # copied during the plan's export, or made on the device, or copied now
                if pd is not None:
                    setattr(self, k, pd[k] if pd[k].numel() else torch.zeros(1, dtype=pd[k].dtype, device=d))
                    if not built_on_device:
                        self.h2d_bytes += pd[k].numel() * pd[k].element_size()
                else:
                    setattr(self, k, up(getattr(plan, k)))
            self.row_vert = up(plan.row_vert); self.vert_row = up(plan.vert_row)
            self.agg_rows = up(plan.agg_rows); self.cofs = up(plan.cofs)
            # geometry
            n, t, nc = max(self.n, 1), max(self.t, 1), max(self.nc, 1)
            f64, f32 = torch.float64, torch.float32
            # asynchronous uploads read page-locked host memory until they finish:
            # the batch keeps its host sources alive (the plan holds the rest)
            self._host_src = (P, U)
            if isinstance(P, torch.Tensor) and P.is_cuda:   # already on the device (uploaded by the caller)
                self.P = P.to(d, f64).reshape(-1, 3)
            else:
                self.P = up(np.asarray(P, np.float64).reshape(-1, 3)) if self.n else torch.zeros((1, 3), dtype=f64, device=d)
            self.frame = torch.empty((t, 4), dtype=f64, device=d)
            self.wtri = torch.empty((t, 4), dtype=f64, device=d)
            self.tscale = torch.ones(t, dtype=f32, device=d)
            self.wedge = torch.empty(max(plan.E, 1), dtype=f64, device=d)
            self.slot_cw = torch.empty((max(plan.nslots, 1), 2), dtype=torch.int32, device=d)
            self.wdiag = torch.empty(n, dtype=f64, device=d)
            nco = max(plan.ncoarse, 1)
            self.coarse_a = torch.empty(nco, dtype=f32, device=d)
            self.coarse_l = torch.empty(4 * nco, dtype=f32, device=d)
            self.coarse_work = torch.empty(4 * nco, dtype=f64, device=d)
            self.cpart = torch.empty(2 * max(plan.nslices, 1), dtype=f32, device=d)
            self.dinv = torch.empty(n, dtype=f32, device=d)
            self.pins = torch.zeros((nc, 3), dtype=torch.int32, device=d)
            self.wpin = torch.empty(nc, dtype=f64, device=d)
            if U is None:
                self.U = torch.zeros((n, 2), dtype=f64, device=d)
            else:
                self.U = up(np.asarray(U, np.float64).reshape(-1, 2)) if self.n else torch.zeros((1, 2), dtype=f64, device=d)
            m = max(n, nc)
            self.x64 = torch.empty((m, 2), dtype=f64, device=d)
            self.b64 = torch.empty((m, 2), dtype=f64, device=d)
            self.rc = torch.empty((t, 3, 2), dtype=f64, device=d)
            self.r32 = torch.empty((n, 2), dtype=f32, device=d)
            self.d32 = torch.empty((n, 2), dtype=f32, device=d)
            self.p32 = torch.empty((n, 2), dtype=f32, device=d)
            self.q32 = torch.empty((n, 2), dtype=f32, device=d)
            self.hist = torch.empty((8, n, 2), dtype=f32, device=d)   # ARAP start history (4 updates, A d)
            self.status = torch.zeros((nc, C.sizeof(_lib.IslandStatus)), dtype=torch.uint8, device=d)
            self.work = torch.zeros(8, dtype=torch.int32, device=d)
            self.rev_ctas = tuned["rev_ctas"] if tuned is not None else 0   # schedule knob (autotune.tune)
        self.desc = self._make_desc()
        self.setup()

    # ------------------------------------------------------------ plumbing
    def _make_desc(self):
        D = _lib.BatchDesc()
        p = self.plan
        D.nc, D.n, D.t, D.E = self.nc, self.n, self.t, p.E
        D.nslices, D.nslots, D.semantics, D.maxrows = p.nslices, p.nslots, self.semantics, p.maxrows
        for c in range(5):
            D.class_ofs[c] = int(p.class_ofs[c])
        for name in ("vofs", "tofs", "sofs", "tri4", "tri_edge", "slice_ptr", "slot_col", "slot_edge", "slot_c",
                     "vt_ptr", "vt", "vflags", "bofs", "bverts", "order", "row_vert", "vert_row", "agg_rows", "cofs",
                     "coarse_a", "coarse_l", "coarse_work", "cpart", "P", "frame", "wtri", "tscale", "wedge",
                     "slot_cw", "wdiag", "dinv", "pins", "wpin", "U", "x64", "b64", "rc", "r32", "d32", "p32",
                     "q32", "status", "work", "hist"):
            setattr(D, name, getattr(self, name).data_ptr())
        return D

    def _refresh_u(self):
        """Re-point the descriptor after U was replaced by a new tensor."""
        self.desc.U = self.U.data_ptr()

    def _stream(self):
        s = self.stream if self.stream is not None else torch.cuda.current_stream(self.dev)
        return C.c_void_p(s.cuda_stream)

    def setup(self):
        check(_lib.lib().uva_batch_setup(C.byref(self.desc), self._stream()), "uva_batch_setup")

    @staticmethod
    def params(kind="arap", iters=1, line_search=True, energy_tol=0.0, threads=0, **over):
        base = dict(DEFAULTS[kind])
        base.update({k: v for k, v in over.items() if v is not None})
        P = _lib.SolveParams()
        P.iters = int(iters); P.line_search = 1 if line_search else 0
        P.tol = float(base["tol"]); P.energy_tol = float(energy_tol)
        P.inner_eta = float(base["inner_eta"]); P.max_inner = int(base["max_inner"])
        P.max_refine = int(base["max_refine"]); P.threads = int(threads)
        P.rev_ctas = int(over.get("rev_ctas") or 0)
        P.fold_step = 1 if over.get("fold_step") else 0
        return P

    # ------------------------------------------------------------ solvers
    def lscm(self, **kw):
        kw.setdefault("rev_ctas", self.rev_ctas)
        prm = self.params("lscm", **kw)
        check(_lib.lib().uva_lscm(C.byref(self.desc), C.byref(prm), self._stream()), "uva_lscm")

    def arap(self, iters=8, line_search=True, energy_tol=0.0, **kw):
        kw.setdefault("rev_ctas", self.rev_ctas)
        prm = self.params("arap", iters=iters, line_search=line_search, energy_tol=energy_tol, **kw)
        check(_lib.lib().uva_arap(C.byref(self.desc), C.byref(prm), self._stream()), "uva_arap")

    def slim(self, iters=10, energy_tol=1e-5, cg_tol=1e-13, cg_max=50000):
        """SLIM iterations of every island (uva_slim; PARAM semantics)."""
        nb = C.c_int64()
        check(_lib.lib().uva_slim_scratch_bytes(C.byref(self.desc), C.byref(nb)), "uva_slim_scratch_bytes")
        scratch = torch.empty(max(int(nb.value) // 8, 2), dtype=torch.float64, device=self.dev)
        prm = self.params("arap", iters=iters, line_search=True, energy_tol=energy_tol, inner_eta=cg_tol,
                          max_inner=cg_max)
        check(_lib.lib().uva_slim(C.byref(self.desc), C.byref(prm), ptr(scratch), self._stream()), "uva_slim")

    def set_classes(self, mid, small):
        """Re-assign islands to team classes (see Plan.set_classes); only the
        work order changes, not the islands' data."""
        self.plan.set_classes(mid, small)
        if self.nc == 0:
            return
        self.order.copy_(torch.from_numpy(self.plan.order).to(self.dev))
        for c in range(5):
            self.desc.class_ofs[c] = int(self.plan.class_ofs[c])

    def step_graph(self, setup=True, lscm=True, arap_iters=20, line_search=True, lscm_kw=None, arap_kw=None):
        """Capture setup + LSCM + ARAP (any subset) into one CUDA graph."""
        return StepGraph(self, setup, lscm, arap_iters, line_search, lscm_kw or {}, arap_kw or {})

    def orient_positive(self):
        check(_lib.lib().uva_orient_positive(C.byref(self.desc), self._stream()), "uva_orient_positive")

    def repair_flips(self, rounds=60, serial=False):
        fn = _lib.lib().uva_repair_flips_serial if serial else _lib.lib().uva_repair_flips
        check(fn(C.byref(self.desc), int(rounds), self._stream()), "uva_repair_flips")

    def flips_per_chart(self):
        out = torch.empty(max(self.nc, 1), dtype=torch.float32, device=self.dev)
        check(_lib.lib().uva_flips_per_chart(C.byref(self.desc), ptr(out), self._stream()), "uva_flips_per_chart")
        return out[:self.nc]

    def signed_area(self, U=None):
        U = self.U if U is None else U.to(self.dev, torch.float64).contiguous()
        out = torch.empty(max(self.t, 1), dtype=torch.float64, device=self.dev)
        check(_lib.lib().uva_signed_area(C.byref(self.desc), ptr(U), ptr(out), self._stream()), "uva_signed_area")
        return out[:self.t]

    def jacobians(self, U=None):
        U = self.U if U is None else U.to(self.dev, torch.float64).contiguous()
        out = torch.empty((max(self.t, 1), 4), dtype=torch.float64, device=self.dev)
        check(_lib.lib().uva_jacobians(C.byref(self.desc), ptr(U), ptr(out), self._stream()), "uva_jacobians")
        return out[:self.t]

    def shrink(self, tri_idx, factor=0.6, floor=0.05, rings=3):
        sel = torch.zeros(max(self.t, 1), dtype=torch.uint8, device=self.dev)
        sel[torch.as_tensor(np.asarray(tri_idx, np.int64), device=self.dev)] = 1
        vmark = torch.empty(max(self.n, 1), dtype=torch.uint8, device=self.dev)
        check(_lib.lib().uva_shrink(C.byref(self.desc), ptr(sel), ptr(vmark), int(rings), float(factor),
                                    float(floor), self._stream()), "uva_shrink")

    def boundary_segments(self):
        """Directed boundary half-edges of every island (rows of U, device
        int32 (nseg, 2)) and their offsets (device (nc + 1,), host copy),
        found once on the device (uva_batch_boundary) and kept."""
        if getattr(self, "_bnd", None) is None:
            L = _lib.lib()
            nb = C.c_int64()
            check(L.uva_batch_boundary_scratch_bytes(C.byref(self.desc), C.byref(nb)), "uva_batch_boundary")
            scratch = torch.empty(max(nb.value, 16), dtype=torch.uint8, device=self.dev)
            sofs = torch.zeros(self.nc + 1, dtype=torch.int32, device=self.dev)
            seg = torch.empty((max(3 * self.t, 1), 2), dtype=torch.int32, device=self.dev)
            check(L.uva_batch_boundary(C.byref(self.desc), ptr(sofs), ptr(seg), ptr(scratch), nb.value,
                                       self._stream()), "uva_batch_boundary")
            sofs_h = sofs.cpu().numpy().astype(np.int64)
            self._bnd = (seg[:int(sofs_h[-1])].clone(), sofs, sofs_h)
        return self._bnd

    def boundary_hits(self, mode=_lib.SEG_COUNT, max_report=1000, U=None):
        """Per island (device int64): mode SEG_COUNT -> the capped boundary
        crossing count of engine/charts.py:596-608 (-1: non-finite UVs);
        SEG_ANY / SEG_ANY_ALL -> 1 if two boundary segments cross."""
        seg, sofs, sofs_h = self.boundary_segments()
        U = self.U if U is None else U.to(self.dev, torch.float64).contiguous()
        L = _lib.lib()
        nseg = int(sofs_h[-1])
        if not hasattr(self, "_bnd_scratch"):
            nb = C.c_int64()
            check(L.uva_seg_scratch_bytes(self.nc, nseg, C.byref(nb)), "uva_seg_scratch_bytes")
            self._bnd_scratch = torch.empty(max(nb.value, 16), dtype=torch.uint8, device=self.dev)
        out = torch.empty(max(self.nc, 1), dtype=torch.int64, device=self.dev)
        d = _lib.SegDesc()
        d.nc, d.nseg, d.n, d.mode = self.nc, nseg, self.n, int(mode)
        d.max_report = int(min(max(int(max_report), -(2 ** 31)), 2 ** 31 - 1))
        d.U, d.vofs, d.seg_ofs = U.data_ptr(), self.vofs.data_ptr(), sofs.data_ptr()
        d.seg = seg.data_ptr() if nseg else None
        d.out, d.scratch, d.scratch_bytes = out.data_ptr(), self._bnd_scratch.data_ptr(), self._bnd_scratch.numel()
        check(L.uva_boundary_hits(C.byref(d), self._stream()), "uva_boundary_hits")
        return out[:self.nc]

    def island_status(self):
        """Per-island solver status (host numpy structured array)."""
        raw = self.status[:self.nc].cpu().numpy()
        dt = np.dtype([("cg_iters", np.int32), ("refinements", np.int32), ("outer_iters", np.int32),
                       ("flags", np.int32), ("resid", np.float64, 2), ("energy", np.float64), ("step", np.float64),
                       ("t_begin", np.int64), ("t_end", np.int64), ("sm", np.int32), ("team", np.int32)])
        return raw.view(dt).reshape(-1)

    def uvs(self):
        """UVs (n, 2) FP64 on the host: one asynchronous copy into
        page-locked memory on the batch's stream, then a wait for it."""
        out = host_empty((self.n, 2), np.float64)
        if self.n:
            s = self.stream if self.stream is not None else torch.cuda.current_stream(self.dev)
            with torch.cuda.stream(s):
                torch.from_numpy(out).copy_(self.U[:self.n], non_blocking=True)
            s.synchronize()
        return out


class StepGraph:
    """A captured batch step (uva_step_graph_create); ``launch()`` replays it
    on the batch's stream. Holds the batch's pointers: rebuild it after the
    batch is re-allocated."""

    def __init__(self, db, setup, lscm, arap_iters, line_search, lscm_kw, arap_kw):
        self.db = db
        parts = (_lib.STEP_SETUP if setup else 0) | (_lib.STEP_LSCM if lscm else 0) | \
                (_lib.STEP_ARAP if arap_iters > 0 else 0)
        lscm_kw = dict(lscm_kw); arap_kw = dict(arap_kw)
        lscm_kw.setdefault("rev_ctas", db.rev_ctas)
        arap_kw.setdefault("rev_ctas", db.rev_ctas)
        self._lp = db.params("lscm", **lscm_kw)
        self._ap = db.params("arap", iters=max(arap_iters, 1), line_search=line_search, **arap_kw)
        h = C.c_void_p()
        check(_lib.lib().uva_step_graph_create(C.byref(db.desc), parts, C.byref(self._lp), C.byref(self._ap),
                                               C.byref(h)), "uva_step_graph_create")
        self._h = h

    def launch(self):
        check(_lib.lib().uva_graph_launch(self._h, self.db._stream()), "uva_graph_launch")

    def close(self):
        if self._h is not None and self._h.value:
            _lib.lib().uva_graph_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
