"""Device mesh bookkeeping behind the drop-in modules: unique edges,
symmetric CSR assembly, CSR products, boundary half-edges, the seam report,
exact corner comparison and segmented sums (``csrc/edges.cu``,
``csrc/report.cu``).

Every function takes and returns torch tensors on a CUDA device (the report
functions take numpy arrays and upload them) and raises ``RuntimeError``
without CUDA: there is no host path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import require_cuda

# element codes of uva_corners_equal
_DTYPE_CODE = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.float16): 2, np.dtype(np.uint8): 3,
               np.dtype(np.int8): 4, np.dtype(np.int16): 5, np.dtype(np.uint16): 6, np.dtype(np.int32): 7,
               np.dtype(np.uint32): 8, np.dtype(np.int64): 9, np.dtype(np.uint64): 10, np.dtype(np.bool_): 11}


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _scratch(nbytes, dev):
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)


def _cuda(t, dtype=None):
    """t on a CUDA device (its own one, else the current one), contiguous."""
    dev = t.device if t.is_cuda else require_cuda()
    return t.to(device=dev, dtype=dtype or t.dtype).contiguous()


def unique_edges(T, n):
    """(ea, eb, inv, cnt) of a triangle list T (t, 3) with vertex ids in
    [0, n): unique undirected edges in ascending (lo, hi) order, the unique
    edge of each of the 3t half-edges (index k t + f: edge of triangle f
    opposite corner k) and the number of triangles using each edge."""
    L = _lib.lib()
    Tc = _cuda(torch.as_tensor(T), torch.int64).reshape(-1, 3)
    dev = Tc.device
    t, n = int(Tc.shape[0]), int(n)
    cap = max(3 * t, 1)
    ea = torch.empty(cap, dtype=torch.int64, device=dev)
    eb = torch.empty_like(ea)
    cnt = torch.empty_like(ea)
    inv = torch.empty(cap, dtype=torch.int64, device=dev)
    ne = torch.zeros(1, dtype=torch.int64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_unique_edges_scratch_bytes(n, t, C.byref(nb)), "uva_unique_edges_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_unique_edges(_p(Tc), t, n, _p(ea), _p(eb), _p(inv), _p(cnt), _p(ne), _p(sc), nb.value,
                                  _stream(dev)), "uva_unique_edges")
    E = int(ne.item())
    if E < 0:
        raise IndexError(f"unique_edges: a vertex id is outside [0, {n})")
    return ea[:E], eb[:E], inv[:3 * t], cnt[:E]


def sym_csr(n, ea, eb, off, diag):
    """n x n symmetric torch CSR tensor (int32 indices, rows sorted by
    column): off[e] at (ea[e], eb[e]) and (eb[e], ea[e]), diag on the
    diagonal. Values are float32 or float64 (the dtype of ``off``)."""
    L = _lib.lib()
    n = int(n)
    off = torch.as_tensor(off)
    vdt = off.dtype if off.dtype in (torch.float32, torch.float64) else torch.float32
    ea = _cuda(torch.as_tensor(ea), torch.int64).reshape(-1)
    dev = ea.device
    eb = torch.as_tensor(eb).to(dev, torch.int64).contiguous().reshape(-1)
    off = off.to(dev, vdt).contiguous().reshape(-1)
    diag = torch.as_tensor(diag).to(dev, vdt).contiguous().reshape(-1)
    ne = int(ea.shape[0])
    if eb.shape[0] != ne or off.shape[0] != ne or diag.shape[0] != n:
        raise ValueError("sym_csr: ea, eb and off need one entry per edge, diag one per row")
    crow = torch.empty(n + 1, dtype=torch.int32, device=dev)
    col = torch.empty(max(2 * ne + n, 1), dtype=torch.int32, device=dev)
    val = torch.empty(max(2 * ne + n, 1), dtype=vdt, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_sym_csr_scratch_bytes(n, C.byref(nb)), "uva_sym_csr_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_sym_csr(n, ne, _p(ea), _p(eb), _p(off), _p(diag), 0 if vdt == torch.float32 else 1, _p(crow),
                             _p(col), _p(val), _p(status), _p(sc), nb.value, _stream(dev)), "uva_sym_csr")
    if int(status.item()):
        raise IndexError(f"sym_csr: an edge endpoint is outside [0, {n})")
    nnz = 2 * ne + n
    return torch.sparse_csr_tensor(crow, col[:nnz], val[:nnz], (n, n))


def csr_spmm(A, X):
    """A @ X for an int32 CSR tensor A and a vector or a few dense columns X,
    all columns in one pass over A."""
    L = _lib.lib()
    crow, col, val = A.crow_indices(), A.col_indices(), A.values()
    if crow.dtype != torch.int32 or col.dtype != torch.int32:
        raise TypeError("csr_spmm: A needs int32 indices (use csr32)")
    if val.dtype not in (torch.float32, torch.float64):
        raise TypeError(f"csr_spmm: unsupported value type {val.dtype}")
    if X.dtype != val.dtype:
        raise RuntimeError(f"csr_spmm: expected X of type {val.dtype}, got {X.dtype}")
    if not val.is_cuda:
        raise RuntimeError("csr_spmm: the matrix must be on a CUDA device")
    dev = val.device
    vec = X.dim() == 1
    Xc = X.reshape(X.shape[0], -1).to(dev).contiguous()
    if Xc.shape[0] != A.shape[1]:
        raise RuntimeError(f"csr_spmm: shapes {tuple(A.shape)} and {tuple(X.shape)} do not match")
    k = int(Xc.shape[1])
    Y = torch.empty((A.shape[0], k), dtype=val.dtype, device=dev)
    _lib.check(L.uva_csr_spmm(int(A.shape[0]), k, int(col.shape[0]), _p(crow), _p(col.contiguous()),
                              _p(val.contiguous()), _p(Xc), _p(Y), 0 if val.dtype == torch.float32 else 1,
                              _stream(dev)), "uva_csr_spmm")
    return Y.reshape(-1) if vec else Y


def boundary_mask(T):
    """bool (3t,) on the device: the directed half-edge k t + f (corners
    k -> k+1 of triangle f) has no reverse half-edge."""
    L = _lib.lib()
    Tc = _cuda(torch.as_tensor(T), torch.int64).reshape(-1, 3)
    dev = Tc.device
    t = int(Tc.shape[0])
    keep = torch.empty(max(3 * t, 1), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_boundary_mask_scratch_bytes(t, C.byref(nb)), "uva_boundary_mask_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_boundary_mask(_p(Tc), t, _p(keep), _p(status), _p(sc), nb.value, _stream(dev)),
               "uva_boundary_mask")
    if int(status.item()):
        raise ValueError("boundary_edges_oriented: vertex ids must lie in [0, 2^31)")
    return keep[:3 * t].bool()


def seam_report(V, F, UV, weld=None):
    """(seam_edges, seam_length, open_boundary_edges, open_boundary_length,
    nonmanifold_edge_groups, surface_area) of a mesh with per-vertex UVs."""
    L = _lib.lib()
    dev = require_cuda()
    Vt = torch.from_numpy(np.ascontiguousarray(V, np.float64).reshape(-1, 3)).to(dev)
    Ft = torch.from_numpy(np.ascontiguousarray(F, np.int64).reshape(-1, 3)).to(dev)
    Ut = torch.from_numpy(np.ascontiguousarray(UV, np.float64).reshape(-1, 2)).to(dev)
    Wt = None if weld is None else torch.from_numpy(np.ascontiguousarray(weld, np.int64).reshape(-1)).to(dev)
    n, m = int(Vt.shape[0]), int(Ft.shape[0])
    if Ut.shape[0] < n or (Wt is not None and Wt.shape[0] < n):
        raise IndexError("seam_report: uvs and weld keys need a row per vertex")
    out = torch.zeros(6, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_seam_report_scratch_bytes(n, m, C.byref(nb)), "uva_seam_report_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_seam_report(_p(Vt), n, _p(Ft), m, _p(Ut), _p(Wt), _p(out), _p(status), _p(sc), nb.value,
                                 _stream(dev)), "uva_seam_report")
    if int(status.item()):
        raise IndexError(f"seam_report: a face index is outside the {n} vertices")
    return out.cpu().numpy()


def _rows(a):
    """(array as rows of w columns, w) for a (n, ...) attribute array."""
    a = np.asarray(a)
    if a.dtype.kind == "b":
        a = a.view(np.uint8)
    return np.ascontiguousarray(a.reshape(len(a), -1)), int(np.prod(a.shape[1:], dtype=np.int64))


def corners_equal(a, fa, b, fb):
    """np.array_equal(a[fa], b[fb]) for attribute arrays a, b (one row per
    vertex) and equal-length corner index arrays fa, fb, on the device.
    Raises IndexError for an index outside its array, as numpy does."""
    fa = np.asarray(fa).reshape(-1)
    fb = np.asarray(fb).reshape(-1)
    a = np.asarray(a)
    b = np.asarray(b)
    if fa.shape != fb.shape or a.shape[1:] != b.shape[1:]:
        return False
    if a.dtype not in _DTYPE_CODE or b.dtype not in _DTYPE_CODE:
        raise TypeError(f"corners_equal: unsupported element types {a.dtype}, {b.dtype}")
    L = _lib.lib()
    dev = require_cuda()
    ar, w = _rows(a)
    br, _ = _rows(b)
    ta = torch.from_numpy(ar).to(dev)
    tb = torch.from_numpy(br).to(dev)
    ia = torch.from_numpy(np.ascontiguousarray(fa, np.int64)).to(dev)
    ib = torch.from_numpy(np.ascontiguousarray(fb, np.int64)).to(dev)
    res = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(L.uva_corners_equal(_p(ta), _DTYPE_CODE[a.dtype], len(ar), _p(ia), _p(tb), _DTYPE_CODE[b.dtype],
                                   len(br), _p(ib), int(fa.shape[0]), w, _p(res), _stream(dev)), "uva_corners_equal")
    r = int(res.item())
    if r & 2:
        raise IndexError("corners_equal: a corner index is outside its array")
    return r == 0


def segment_sum(x, seg, nseg, stride=1):
    """Device float64 (nseg,): sum of x[i * stride] over i with seg[i] == g."""
    L = _lib.lib()
    dev = x.device
    seg = seg.to(dev, torch.int32).contiguous()
    out = torch.zeros(max(int(nseg), 1), dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(L.uva_segment_sum(_p(x), int(stride), _p(seg), int(seg.shape[0]), int(nseg), _p(out), _p(status),
                                 _stream(dev)), "uva_segment_sum")
    if int(status.item()):
        raise IndexError("segment_sum: a segment id is outside [0, nseg)")
    return out[:int(nseg)]
