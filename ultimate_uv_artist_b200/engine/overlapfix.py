"""Drop-in replacement of the per-chart overlap checks of the reference's
``engine/overlapfix.py``: ``overlapping_triangles`` (:212-224),
``raster_overlap`` (:263-275) and ``collision`` (:283-296), with the
reference's signatures and results.

* ``overlapping_triangles`` / ``raster_overlap``: the texel-centre raster of
  the chart normalised like the reference ((U - lo) / ext * 0.999, the
  resolution from the triangle count), on the GPU (uva_overlap_raster): every
  texel gets its coverage count and its first (smallest) triangle. A
  triangle overlaps when a texel it covers has two coverers, which is what
  the reference's serial owner raster marks. The first pair is the smallest
  triangle that meets a texel an earlier one owns, paired with that texel's
  owner at the first such texel of its scan.
* ``collision``: the first crossing pair of boundary segments in the
  reference's cell scan (uva_boundary_hits, mode FIRST), mapped to the
  triangles that own the two segments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib, segments
from ..device import require_cuda


def _raster(U, T, res, want_pair, dev=None):
    dev = require_cuda(dev)
    L = _lib.lib()
    U = np.asarray(U, np.float64).reshape(-1, 2)
    T = np.asarray(T, np.int64).reshape(-1, 3)
    lo = U.min(0)
    ext = float((U.max(0) - lo).max())
    uv = np.ascontiguousarray((U - lo) / ext * 0.999, np.float64)
    m = len(T)
    if T.min() < 0 or T.max() >= len(U):
        raise IndexError("overlapfix: T names a vertex outside U")
    uvd = torch.from_numpy(uv).to(dev)
    Fd = torch.from_numpy(T.astype(np.int32)).to(dev)
    nb = C.c_int64()
    _lib.check(L.uva_gutter_scratch_bytes(int(res), m, C.byref(nb)), "uva_gutter_scratch_bytes")
    scratch = torch.empty(max(nb.value, 16), dtype=torch.uint8, device=dev)
    flags = torch.empty(max(m, 1), dtype=torch.uint8, device=dev)
    pair = torch.empty(2, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    _lib.check(L.uva_overlap_raster(uvd.data_ptr(), Fd.data_ptr(), m, int(res), flags.data_ptr(),
                                    pair.data_ptr() if want_pair else None, scratch.data_ptr(), nb.value,
                                    C.c_void_p(st.cuda_stream)), "uva_overlap_raster")
    return flags[:m].cpu().numpy().astype(bool), pair.cpu().numpy()


def _degenerate(U, T):
    if len(T) < 2:
        return True
    U = np.asarray(U, np.float64).reshape(-1, 2)
    lo = U.min(0)
    ext = float((U.max(0) - lo).max())
    return not np.isfinite(ext) or ext <= 0


def overlapping_triangles(U, T, res=None):
    """Bool per triangle: involved in a UV overlap (texel-centre raster)
    (engine/overlapfix.py:212-224)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if _degenerate(U, T):
        return np.zeros(len(T), np.bool_)
    if res is None:
        res = int(np.clip(np.sqrt(len(T)) * 2.5, 64, 3072))
    flags, _ = _raster(U, T, res, False)
    return flags


def raster_overlap(U, T, res=None):
    """Triangles (ta, tb) overlapping in UV (texel-centre raster), or None
    (engine/overlapfix.py:263-275)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    if _degenerate(U, T):
        return None
    if res is None:
        res = int(np.clip(np.sqrt(len(T)) * 2.0, 64, 2048))
    _, pair = _raster(U, T, res, True)
    return None if pair[0] < 0 else (int(pair[0]), int(pair[1]))


def _boundary_with_faces(T):
    """Directed boundary half-edges and the triangle owning each, face by face
    (engine/overlapfix.py:16-41)."""
    T = np.asarray(T, np.int64).reshape(-1, 3)
    a = T.reshape(-1)
    b = T[:, [1, 2, 0]].reshape(-1)
    fo = np.repeat(np.arange(len(T), dtype=np.int64), 3)
    if len(a) == 0:
        return a, b, fo
    n = int(T.max()) + 1
    keep = ~np.isin(b * n + a, a * n + b)
    return a[keep], b[keep], fo[keep]


def collision(U, T):
    """Local triangle indices (fa, fb) owning two crossing boundary edges, or
    None (engine/overlapfix.py:283-296): the first pair the reference's cell
    scan meets."""
    U = np.asarray(U, np.float64).reshape(-1, 2)
    a, b, fo = _boundary_with_faces(T)
    if len(a) < 3:
        return None
    out = segments.boundary_hits(U, [0, len(a)], np.stack([a, b], 1), segments.FIRST, vofs=[0, len(U)])
    r = int(out[0])
    if r == -1:
        raise ValueError("collision: non-finite UVs")
    if r < 0:
        if r == -2:
            raise IndexError("collision: T names a vertex outside U")
        return None
    return int(fo[r >> 32]), int(fo[r & 0xffffffff])
