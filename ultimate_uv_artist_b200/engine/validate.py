"""Drop-in replacement of the reference's ``engine/validate.py``.

``validate_uvs`` and ``chart_overlaps`` keep the reference's signatures and
report keys (engine/validate.py:139-226). Every check runs in the uva_b200
CUDA kernels on float32-rounded UVs with FP64 predicates compiled without
FMA contraction, so the verdicts match the reference bit for bit:

* range and non-finite counts per UV row;
* degenerate and sub-float32 sliver triangles;
* islands (vertices welded by identical float32 position + UV bytes);
* flips against each island's dominant orientation and mirrored islands
  (near-tied orientation sums are re-summed in the reference's face order);
* exact positive-area overlaps (tolerant) and float32 contacts (strict),
  binned on a uniform grid;
* the gutter (conservative raster, exact Euclidean distance transform).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib, meshops
from ..device import require_cuda

ULP = 2.0 ** -24
ULP_STRICT = 0.0

(VC_NONFINITE, VC_OUTSIDE, VC_DEGENERATE, VC_SLIVERS, VC_FLIPPED, VC_MIRRORED, VC_ISLANDS, VC_OVERLAP,
 VC_CONTACTS, VC_ISLANDS_OV, VC_PAIRS, VC_BIG, VC_AMBIGUOUS) = range(13)
VC_N = 16


class ValDesc(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("grid", C.c_int32), ("reserved", C.c_int32),
                ("V", C.c_void_p), ("UV", C.c_void_p), ("F", C.c_void_p), ("rel", C.c_double),
                ("tflags", C.c_void_p), ("labels", C.c_void_p), ("sa", C.c_void_p), ("counts", C.c_void_p),
                ("scratch", C.c_void_p), ("scratch_bytes", C.c_int64), ("shard", C.c_int32), ("nshards", C.c_int32)]


def _sig():
    L = _lib.lib()
    if not getattr(L, "_uva_val_sig", False):
        L.uva_validate.argtypes = [C.c_void_p, C.c_void_p]
        L.uva_validate.restype = C.c_int32
        L.uva_validate_scratch_bytes.argtypes = [C.c_int64, C.c_int64, C.c_int32, C.c_void_p]
        L.uva_validate_scratch_bytes.restype = C.c_int32
        L._uva_val_sig = True
    return L


class DeviceValidation:
    """One validation pass on the device; results stay on the device until read."""

    def __init__(self, V, F, UV32, rel=1e-6, grid=0, device=None, stream=None, shard=0, nshards=1):
        L = _sig()
        self.dev = require_cuda(device)
        d = self.dev
        self.n, self.m = int(V.shape[0]), int(F.shape[0])
        self.V = V if torch.is_tensor(V) else torch.from_numpy(np.ascontiguousarray(V, np.float64)).to(d)
        self.UV = UV32 if torch.is_tensor(UV32) else torch.from_numpy(np.ascontiguousarray(UV32, np.float32)).to(d)
        self.F = F if torch.is_tensor(F) else torch.from_numpy(np.ascontiguousarray(F, np.int32)).to(d)
        m4 = (max(self.m, 1) + 3) // 4 * 4
        self.tflags = torch.zeros(m4, dtype=torch.uint8, device=d)
        self.labels = torch.zeros(max(self.m, 1), dtype=torch.int32, device=d)
        self.sa = torch.zeros(max(self.m, 1), dtype=torch.float64, device=d)
        self.counts = torch.zeros(VC_N, dtype=torch.int64, device=d)
        nb = C.c_int64()
        _lib.check(L.uva_validate_scratch_bytes(self.n, self.m, int(grid), C.byref(nb)), "uva_validate_scratch_bytes")
        self.scratch = torch.empty(max(int(nb.value), 256), dtype=torch.uint8, device=d)
        D = ValDesc()
        D.n, D.m, D.grid = self.n, self.m, int(grid)
        D.V, D.UV, D.F = self.V.data_ptr(), self.UV.data_ptr(), self.F.data_ptr()
        D.rel = float(rel)
        D.tflags, D.labels, D.sa, D.counts = (self.tflags.data_ptr(), self.labels.data_ptr(), self.sa.data_ptr(),
                                              self.counts.data_ptr())
        D.scratch, D.scratch_bytes = self.scratch.data_ptr(), int(nb.value)
        D.shard, D.nshards = int(shard), int(nshards)
        self.desc = D
        self.stream = stream

    def run(self):
        s = self.stream if self.stream is not None else torch.cuda.current_stream(self.dev)
        _lib.check(_sig().uva_validate(C.byref(self.desc), C.c_void_p(s.cuda_stream)), "uva_validate")
        return self

    def merge(self, group=None):
        """Several shards (one per rank of `group`, each validating its band
        of cell rows): OR the overlap bits of every rank into tflags, sum the
        candidate-pair counts, and recount what depends on the bits
        (uva_validate_finish). Every rank ends with the whole report."""
        from .. import shard as S
        m = self.m
        if m:
            bits = self.tflags[:m]
            ov = S.allreduce_max(((bits & 16) != 0).to(torch.uint8), group)
            st = S.allreduce_max(((bits & 32) != 0).to(torch.uint8), group)
            self.tflags[:m] = (bits & 207) | (ov * 16) | (st * 32)
        self.counts[VC_PAIRS:VC_PAIRS + 1] = S.allreduce_sum(self.counts[VC_PAIRS:VC_PAIRS + 1].clone(), group)
        return self.finish()

    def finish(self):
        """Recount the overlap-dependent counts from tflags after the bits of
        other shards were merged into it (uva_validate_finish)."""
        s = self.stream if self.stream is not None else torch.cuda.current_stream(self.dev)
        _lib.check(_lib.lib().uva_validate_finish(C.byref(self.desc), C.c_void_p(s.cuda_stream)), "uva_validate_finish")
        return self

    def host_counts(self):
        return self.counts.cpu().numpy()

    def flags(self):
        return self.tflags[:self.m].cpu().numpy()


def validate_uvs(v, f, uv, atlas=4096, padding=None, in_v=None, in_f=None, in_normals=None, out_normals=None,
                 in_colors=None, out_colors=None, xref=None, gutter=True, group=None):
    """Checks on final UVs (engine/validate.py:139-209). Returns (report, per-triangle problem mask).

    group: a torch.distributed process group over several GPUs (one rank
    each, every rank holding the whole mesh): each rank tests the overlap
    pairs of its band of the atlas, the overlap bits and pair counts are
    all-reduced, and every rank returns the same report."""
    v = np.asarray(v, np.float64)
    f = np.asarray(f, np.int64)
    uv32 = np.asarray(uv, np.float32)
    from .. import shard as S
    rank, world = S.rank_world(group)
    dv = DeviceValidation(v, f.astype(np.int32), uv32, shard=rank, nshards=world).run()
    if world > 1:
        dv.merge(group)
    c = dv.host_counts()
    fl = dv.flags()
    rep = {}
    rep["non_finite_uv"] = int(c[VC_NONFINITE])
    rep["uv_outside_unit_square"] = int(c[VC_OUTSIDE])
    rep["degenerate_uv_triangles"] = int(c[VC_DEGENERATE])
    rep["sub_float32_slivers"] = int(c[VC_SLIVERS])
    rep["flipped_triangles"] = int(c[VC_FLIPPED])
    rep["mirrored_islands"] = int(c[VC_MIRRORED])
    rep["islands"] = int(c[VC_ISLANDS])
    rep["overlapping_triangles_exact"] = int(c[VC_OVERLAP])
    rep["float32_contacts"] = int(c[VC_CONTACTS])
    if c[VC_OVERLAP] > 0:
        rep["islands_with_overlap"] = int(c[VC_ISLANDS_OV])
    if gutter:
        from . import metrics
        res = min(atlas, 8192)
        g = metrics.min_gutter_device(dv.UV.double(), dv.F, dv.labels, int(c[VC_ISLANDS]), res)
        rep["min_gutter_texels"] = float(g * atlas / res)
        if padding is not None:
            rep["gutter_ok"] = bool(rep["min_gutter_texels"] >= padding - 1e-6)
    if in_v is not None and in_f is not None:
        in_v = np.asarray(in_v, np.float64)
        in_f = np.asarray(in_f, np.int64)
        rep["triangle_count_preserved"] = bool(len(in_f) == len(f))
        if len(in_f) == len(f):
            rep["corner_positions_exact"] = _corners_equal(np.asarray(v, np.float32), f, np.asarray(in_v, np.float32), in_f)
            if in_normals is not None and out_normals is not None:
                rep["corner_normals_exact"] = _corners_equal(np.asarray(out_normals), f, np.asarray(in_normals), in_f)
            if in_colors is not None and out_colors is not None:
                rep["corner_colors_exact"] = _corners_equal(np.asarray(out_colors), f, np.asarray(in_colors), in_f)
    problems = (fl & (16 | 8)) != 0
    bad = rep["non_finite_uv"] + rep["uv_outside_unit_square"] + rep["flipped_triangles"] + rep["overlapping_triangles_exact"]
    if gutter and padding is not None and not rep.get("gutter_ok", True):
        bad += 1
    for k in ("triangle_count_preserved", "corner_positions_exact", "corner_normals_exact", "corner_colors_exact"):
        if rep.get(k) is False:
            bad += 1
    rep["valid"] = bool(bad == 0)
    return rep, problems


def _corners_equal(a, fa, b, fb):
    """np.array_equal(a[fa], b[fb]) (engine/validate.py:195-199), compared on
    the device by uva_corners_equal."""
    return meshops.corners_equal(a, fa, b, fb)


def chart_overlaps(U, T):
    """Exact positive-area self-overlap of one chart in any UV units
    (engine/validate.py:212-226). Returns a bool per triangle."""
    U = np.asarray(U, np.float64)
    T = np.ascontiguousarray(T, np.int64)
    if len(T) < 2:
        return np.zeros(len(T), np.bool_)
    lo = U.min(0)
    ext = float((U.max(0) - lo).max())
    if not np.isfinite(ext) or ext <= 0:
        return np.zeros(len(T), np.bool_)
    Un = np.ascontiguousarray((U - lo) / ext * 0.999999)
    flags = _chart_overlap_flags(Un, T)
    return flags


def _chart_overlap_flags(Un, T):
    """Overlap flags of one normalised chart: the validation kernels with the
    chart's skip rule |sa| <= 1e-14 (engine/validate.py:223-226)."""
    L = _sig()
    if not getattr(L, "_uva_chart_sig", False):
        L.uva_chart_overlaps.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.c_void_p]
        L.uva_chart_overlaps.restype = C.c_int32
        L._uva_chart_sig = True
    dev = require_cuda()
    n, m = len(Un), len(T)
    U = torch.from_numpy(Un).to(dev)
    F = torch.from_numpy(T.astype(np.int32)).to(dev)
    out = torch.zeros((m + 3) // 4 * 4, dtype=torch.uint8, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_validate_scratch_bytes(n, m, 0, C.byref(nb)), "uva_validate_scratch_bytes")
    scratch = torch.empty(max(int(nb.value), 256), dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream(dev)
    _lib.check(L.uva_chart_overlaps(C.c_void_p(U.data_ptr()), C.c_void_p(F.data_ptr()), n, m, C.c_void_p(out.data_ptr()),
                                    C.c_void_p(scratch.data_ptr()), int(nb.value), C.c_void_p(s.cuda_stream)),
               "uva_chart_overlaps")
    return (out[:m].cpu().numpy() & 16) != 0
