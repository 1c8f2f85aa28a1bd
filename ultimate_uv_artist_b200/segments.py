"""Host side of the batched boundary self-intersection checks (uva_boundary_hits).

``boundary_hits`` takes host or device arrays: UV rows, the charts' row
ranges (count mode) and their directed boundary segments grouped by chart,
and returns one int64 per chart, computed on the GPU. The callers are
``engine.charts`` (boundary_intersections) and ``engine.hier``
(charts_collide, chart_checks).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import require_cuda

COUNT, ANY, ANY_ALL, FIRST = _lib.SEG_COUNT, _lib.SEG_ANY, _lib.SEG_ANY_ALL, _lib.SEG_FIRST


def _dev_array(a, dtype, dev):
    t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
    return t.to(dev, dtype).contiguous()


def boundary_hits(U, seg_ofs, seg, mode, max_report=1000, vofs=None, device=None, stream=None):
    """Per chart: COUNT -> the reference's capped crossing count (-1: non-finite
    UVs with >= 3 segments, -2: a segment row outside its chart); ANY -> 1 if
    two segments cross (or the extent is not below 1e300), else 0; ANY_ALL ->
    1 if two segments cross.

    U (n, 2) UVs (FP64 on the device), seg_ofs (nc + 1), seg (nseg, 2) rows
    of U, vofs (nc + 1) the charts' UV rows (COUNT only). Returns numpy int64 (nc,).
    """
    dev = require_cuda(device)
    L = _lib.lib()
    seg_ofs = np.ascontiguousarray(seg_ofs, np.int64)
    nc = len(seg_ofs) - 1
    if nc <= 0:
        return np.zeros(0, np.int64)
    seg = np.asarray(seg).reshape(-1, 2) if not isinstance(seg, torch.Tensor) else seg.reshape(-1, 2)
    nseg = int(seg.shape[0])
    Ud = _dev_array(U, torch.float64, dev).reshape(-1, 2)
    n = int(Ud.shape[0])
    if max(n, nseg, int(seg_ofs[-1])) >= 2 ** 31:
        raise ValueError("boundary_hits: more than 2^31 - 1 rows or segments")
    if mode in (COUNT, FIRST) and vofs is None:
        raise ValueError("boundary_hits: count mode needs the charts' UV rows (vofs)")
    seg_d = _dev_array(seg, torch.int32, dev) if nseg else torch.zeros((1, 2), dtype=torch.int32, device=dev)
    ofs_d = _dev_array(seg_ofs, torch.int32, dev)
    vofs_d = _dev_array(np.asarray(vofs, np.int64), torch.int32, dev) if vofs is not None else None
    if n == 0:
        Ud = torch.zeros((1, 2), dtype=torch.float64, device=dev)
    out = torch.empty(nc, dtype=torch.int64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_seg_scratch_bytes(nc, nseg, C.byref(nb)), "uva_seg_scratch_bytes")
    scratch = torch.empty(max(nb.value, 16), dtype=torch.uint8, device=dev)
    d = _lib.SegDesc()
    d.nc, d.nseg, d.n, d.mode = nc, nseg, n, int(mode)
    d.max_report = int(min(max(int(max_report), -(2 ** 31)), 2 ** 31 - 1))
    d.U = Ud.data_ptr()
    d.vofs = vofs_d.data_ptr() if vofs_d is not None else None
    d.seg_ofs = ofs_d.data_ptr()
    d.seg = seg_d.data_ptr()
    d.out = out.data_ptr()
    d.scratch = scratch.data_ptr()
    d.scratch_bytes = nb.value
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    _lib.check(L.uva_boundary_hits(C.byref(d), C.c_void_p(st.cuda_stream)), "uva_boundary_hits")
    return out.cpu().numpy()


def directed_boundary(T):
    """Directed half-edges (a -> b) of a triangle list whose reverse (b -> a)
    is absent, with the index of the triangle each one belongs to
    (engine/param.py:59-68, which lists them corner-major)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]])
    b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
    tri = np.tile(np.arange(len(T), dtype=np.int64), 3)
    if len(a) == 0:
        return a, b, tri
    n = int(max(a.max(), b.max())) + 1
    keep = ~np.isin(b * n + a, a * n + b)
    return a[keep], b[keep], tri[keep]
