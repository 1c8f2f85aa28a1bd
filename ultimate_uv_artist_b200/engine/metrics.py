"""Drop-in replacement of the reference's ``engine/metrics.py``.

Same functions and signatures (engine/metrics.py:13-373). Distortion
(Jacobian singular values, anisotropy, density and chart-area ratios, angle
error, weighted p95 quantiles), islands, coverage and label rasters, the
gutter, the seam report (vertex weld and edge grouping by hash tables) and
the exact corner comparison of the preservation report run in the uva_b200
CUDA kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib, meshops
from ..device import require_cuda, to_host

vp = C.c_void_p


def _sig():
    L = _lib.lib()
    if getattr(L, "_uva_met_sig", False):
        return L
    sigs = {
        "uva_islands": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_int64, vp]),
        "uva_validate_scratch_bytes": ([C.c_int64, C.c_int64, C.c_int32, vp]),
        "uva_gutter_scratch_bytes": ([C.c_int32, C.c_int64, vp]),
        "uva_gutter": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_int64, vp, vp]),
        "uva_raster_counts": ([vp, vp, C.c_int32, C.c_int32, vp, vp, vp, C.c_int64, vp]),
        "uva_metrics_scratch_bytes": ([C.c_int64, C.c_int64, vp]),
        "uva_distortion_report": ([vp, vp, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_int64, vp]),
        "uva_wquantile_scratch_bytes": ([C.c_int32, vp]),
        "uva_wquantile": ([vp, vp, vp, C.c_int32, C.c_int32, C.c_double, vp, vp, C.c_int64, vp]),
    }
    for k, a in sigs.items():
        fn = getattr(L, k)
        fn.argtypes = a
        fn.restype = C.c_int32
    L._uva_met_sig = True
    return L


def _p(t):
    return C.c_void_p(t.data_ptr())


def _stream(dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _scratch(nbytes, dev):
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)


# ---------------------------------------------------------------- rasterizer
def _raster_counts(uv, faces, res, counts):
    """Coverage counts per texel centre, top-left rule (engine/metrics.py:13-54).
    Fills ``counts`` (res x res uint8) in place, like the reference."""
    c, _ = _raster_counts_device(uv, faces, int(res))
    counts[...] = np.minimum(counts.astype(np.int32) + c.astype(np.int32), 255).astype(counts.dtype)


def _raster_counts_device(uv, faces, res):
    L = _sig()
    dev = require_cuda()
    U = torch.from_numpy(np.ascontiguousarray(uv, np.float64)).to(dev)
    F = torch.from_numpy(np.ascontiguousarray(faces, np.int32).reshape(-1, 3)).to(dev)
    m = int(F.shape[0])
    out = torch.empty((res, res), dtype=torch.uint8, device=dev)
    stats = torch.zeros(2, dtype=torch.int64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_gutter_scratch_bytes(res, m, C.byref(nb)), "uva_gutter_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_raster_counts(_p(U), _p(F), m, res, _p(out), _p(stats), _p(sc), nb.value, _stream(dev)),
               "uva_raster_counts")
    return out.cpu().numpy(), stats.cpu().numpy()


def raster_coverage(uv, faces, res=4096):
    """engine/metrics.py:57-62: (counts, covered fraction, overlap texels)."""
    counts, stats = _raster_counts_device(uv, faces, int(res))
    return counts, int(stats[0]) / float(res * res), int(stats[1])


# ---------------------------------------------------------------- islands
def uv_islands(faces, n_vertices, uv=None, vertices=None):
    """Face islands (engine/metrics.py:91-103). With ``uv`` and ``vertices``,
    vertices with identical float32 position and UV are one vertex. Labels are
    0..n-1 by the smallest (representative) vertex of each island; the
    partition equals the reference's."""
    L = _sig()
    dev = require_cuda()
    F = torch.from_numpy(np.ascontiguousarray(faces, np.int32).reshape(-1, 3)).to(dev)
    m = int(F.shape[0])
    n = int(n_vertices)
    weld = uv is not None and vertices is not None
    if weld:
        V = torch.from_numpy(np.ascontiguousarray(vertices, np.float64).reshape(-1, 3)).to(dev)
        UV = torch.from_numpy(np.ascontiguousarray(uv, np.float32).reshape(-1, 2)).to(dev)
        n = int(V.shape[0])
    else:
        V = UV = None
    labels = torch.zeros(max(m, 1), dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_validate_scratch_bytes(n, m, 0, C.byref(nb)), "uva_validate_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_islands(_p(V) if weld else None, _p(UV) if weld else None, _p(F), n, m, 1 if weld else 0,
                             _p(labels), _p(count), _p(sc), nb.value, _stream(dev)), "uva_islands")
    return labels[:m].cpu().numpy().astype(np.int32), int(count.item())


# ---------------------------------------------------------------- distortion
def _wquantile(x, w, q):
    """Area-weighted quantile (engine/metrics.py:107-112) on the device."""
    L = _sig()
    dev = require_cuda()
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    if len(x) == 0:
        return float("nan")
    X = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    W = torch.from_numpy(np.ascontiguousarray(w)).to(dev)
    out = torch.empty(1, dtype=torch.float64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_wquantile_scratch_bytes(1, C.byref(nb)), "uva_wquantile_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_wquantile(_p(X), _p(W), None, len(x), 1, float(q), _p(out), _p(sc), nb.value, _stream(dev)),
               "uva_wquantile")
    return float(out.item())


def triangle_jacobians(P, U):
    """P: (F,3,3) 3D corners, U: (F,3,2) UV corners -> s1, s2, signed UV area,
    3D area, good (engine/metrics.py:115-145)."""
    P = np.asarray(P, np.float64).reshape(-1, 3, 3)
    U = np.asarray(U, np.float64).reshape(-1, 3, 2)
    m = len(P)
    F = np.arange(3 * m, dtype=np.int32).reshape(-1, 3)
    per = _distortion(P.reshape(-1, 3), F, U.reshape(-1, 2), None, 0)[1]
    return per[:, 0], per[:, 1], per[:, 2], per[:, 3], per[:, 4] != 0


def _distortion(V, F, UV, islands, n_islands, per_tri="host", keep_per_tri=False):
    """One uva_distortion_report pass: (report sums on the host, per-triangle
    s1, s2, signed UV area, 3D area, good, angle error). per_tri "host":
    numpy; with keep_per_tri the device tensor is returned instead; None:
    not written (the kernel keeps it in its scratch)."""
    L = _sig()
    dev = require_cuda()
    Vt = torch.from_numpy(np.ascontiguousarray(V, np.float64).reshape(-1, 3)).to(dev)
    Ft = torch.from_numpy(np.ascontiguousarray(F, np.int32).reshape(-1, 3)).to(dev)
    Ut = torch.from_numpy(np.ascontiguousarray(UV, np.float64).reshape(-1, 2)).to(dev)
    It = torch.from_numpy(np.ascontiguousarray(islands, np.int32)).to(dev) if islands is not None else None
    m = int(Ft.shape[0])
    out = torch.zeros(32, dtype=torch.float64, device=dev)
    want = keep_per_tri or per_tri is not None
    per = torch.empty((max(m, 1), 6), dtype=torch.float64, device=dev) if want else None
    nb = C.c_int64()
    _lib.check(L.uva_metrics_scratch_bytes(m, int(n_islands), C.byref(nb)), "uva_metrics_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_distortion_report(_p(Vt), _p(Ut), _p(Ft), _p(It) if It is not None else None, int(Vt.shape[0]),
                                       m, int(n_islands), _p(out), _p(per) if want else None, _p(sc), nb.value,
                                       _stream(dev)),
               "uva_distortion_report")
    if keep_per_tri:
        return out.cpu().numpy(), per[:m]
    return out.cpu().numpy(), (to_host(per[:m]) if want else None)


def _distortion_fields(m, s, with_islands):
    """The report dictionary of distortion_report from the pass's sums."""
    out = {}
    out["triangles"] = int(m)
    out["collapsed_uv_triangles"] = int(round(s[2]))
    out["collapsed_uv_area_fraction"] = float(s[3])
    out["anisotropy_mean"] = float(s[4] / max(s[5], 1e-30))
    out["anisotropy_p95"] = float(s[24])
    out["angle_error_deg_mean"] = float(s[6] / max(s[7], 1e-30))
    out["density_log2_dev_mean"] = float(s[8] / max(s[9], 1e-30))
    out["density_ratio_p95"] = float(2 ** s[25])
    out["stretch_L2"] = float(np.sqrt(s[10] / max(s[9], 1e-30)))
    if with_islands:
        out["chart_area_log2_dev_mean"] = float(s[11] / max(s[9], 1e-30))
        out["chart_area_ratio_p95"] = float(2 ** s[26])
        out["flipped_triangles"] = int(round(s[12]))
        out["flipped_area_fraction"] = float(s[13])
        out["mirrored_islands"] = int(round(s[16]))
        out["island_density_ratio_p95"] = float(2 ** s[27])
    return out


def distortion_report(vertices, faces, uvs, islands=None, chunk=2_000_000):
    """Area-weighted distortion statistics (engine/metrics.py:148-210).
    ``chunk`` is accepted for signature compatibility (the device holds the
    whole mesh)."""
    faces = np.asarray(faces, np.int64)
    n_is = int(np.asarray(islands).max()) + 1 if islands is not None and len(islands) else 0
    s, _ = _distortion(vertices, faces, uvs, islands, n_is, per_tri=None)
    return _distortion_fields(len(faces), s, islands is not None)


def _angle_error(P, U):
    """Mean absolute corner-angle difference in degrees (engine/metrics.py:213-223)."""
    P = np.asarray(P, np.float64).reshape(-1, 3, 3)
    U = np.asarray(U, np.float64).reshape(-1, 3, 2)
    F = np.arange(3 * len(P), dtype=np.int32).reshape(-1, 3)
    return _distortion(P.reshape(-1, 3), F, U.reshape(-1, 2), None, 0)[1][:, 5]


# ---------------------------------------------------------------- seams and preservation
def seam_report(vertices, faces, uvs, weld_keys=None):
    """UV seam edges and lengths (engine/metrics.py:227-261), on the device
    (``uva_seam_report``): vertices weld by equal position (or by equal
    ``weld_keys``), the triangle edges of the welded mesh are grouped, and a
    group of two whose corners disagree on UVs is a seam edge; groups of one
    are open boundary, of more than two non-manifold."""
    s = meshops.seam_report(vertices, faces, uvs, weld_keys)
    seam_len, area = float(s[1]), float(s[5])
    return {"seam_edges": int(s[0]), "seam_length": seam_len,
            "seam_length_per_sqrt_area": float(seam_len / np.sqrt(max(area, 1e-30))),
            "open_boundary_edges": int(s[2]), "open_boundary_length": float(s[3]),
            "nonmanifold_edge_groups": int(s[4]), "surface_area": area}


def preservation_report(in_v, in_f, out_v, out_f, in_attrs=None, out_attrs=None, chunk=2_000_000):
    """Exact per-corner equality of positions and attributes between the
    input and output meshes (engine/metrics.py:264-286), compared on the
    device (``uva_corners_equal``). ``chunk`` is accepted for signature
    compatibility: the device compares all corners in one launch."""
    same_count = len(in_f) == len(out_f)
    rep = {"triangle_count_equal": same_count}
    if not same_count:
        rep["positions_exact"] = False
        return rep
    rep["positions_exact"] = meshops.corners_equal(in_v, in_f, out_v, out_f)
    out_attrs = out_attrs or {}
    for name, a in (in_attrs or {}).items():
        if a is None:
            continue
        o = out_attrs.get(name)
        rep[name + "_exact"] = False if o is None else meshops.corners_equal(a, in_f, o, out_f)
    return rep


def full_report(out_v, out_f, out_uv, raster_res=4096, in_v=None, in_f=None, in_attrs=None, out_attrs=None):
    """Islands, coverage, distortion, seams, preservation and the island size
    distribution of an unwrapped mesh (engine/metrics.py:289-311). Returns
    (report, per-face island labels)."""
    out_f = np.asarray(out_f)
    isl, n_is = uv_islands(out_f, len(out_v), out_uv, out_v)
    rep = {"islands": n_is}
    uv = np.asarray(out_uv)
    rep["uv_finite"] = bool(np.isfinite(uv).all())
    rep["uv_in_unit_square"] = bool(uv.min() >= -1e-6 and uv.max() <= 1 + 1e-6)
    _, occ, ov = raster_coverage(out_uv, out_f, raster_res)
    rep["raster_res"] = raster_res
    rep["occupancy"] = occ
    rep["overlap_texels"] = ov
    sums, per = _distortion(out_v, out_f, out_uv, isl, n_is, keep_per_tri=True)
    rep.update(_distortion_fields(len(out_f), sums, True))
    rep.update(seam_report(out_v, out_f, out_uv))
    if in_v is not None:
        rep.update(preservation_report(in_v, in_f, out_v, out_f, in_attrs, out_attrs))
    # island 3D areas (the distortion pass's per-triangle areas summed per
    # island), largest first, as fractions of the total
    if n_is:
        ia = meshops.segment_sum(per[:, 3].contiguous(), torch.from_numpy(np.asarray(isl, np.int32)), n_is)
        ia = np.sort(ia.cpu().numpy())[::-1]
        ia = ia / max(float(ia.sum()), 1e-30)
        rep["largest_island_area_frac"] = float(ia[0])
        rep["islands_for_90pct_area"] = int(np.searchsorted(np.cumsum(ia), 0.9) + 1)
        rep["tiny_islands_lt_0.01pct"] = int((ia < 1e-4).sum())
    else:
        rep["largest_island_area_frac"] = 0.0
        rep["islands_for_90pct_area"] = 0
        rep["tiny_islands_lt_0.01pct"] = 0
    return rep, isl


# ---------------------------------------------------------------- gutters
def _raster_labels(uv, faces, lab_of_face, res, img):
    """Conservative label raster, last triangle wins (engine/metrics.py:315-345);
    fills ``img`` (res x res int32) in place."""
    L = _sig()
    dev = require_cuda()
    UV = torch.from_numpy(np.ascontiguousarray(uv, np.float64)).to(dev)
    F = torch.from_numpy(np.ascontiguousarray(faces, np.int32).reshape(-1, 3)).to(dev)
    lab = torch.from_numpy(np.ascontiguousarray(lab_of_face, np.int32)).to(dev)
    out, _ = _gutter_raw(UV, F, lab, int(res), 1)
    res_img = to_host(out)
    np.copyto(img, np.where(res_img >= 0, res_img, img))


def _gutter_raw(UV, F, labels, res, radius):
    L = _sig()
    dev = UV.device
    m = int(F.shape[0])
    img = torch.empty((res, res), dtype=torch.int32, device=dev)
    out = torch.empty(4, dtype=torch.float64, device=dev)
    nb = C.c_int64()
    _lib.check(L.uva_gutter_scratch_bytes(res, m, C.byref(nb)), "uva_gutter_scratch_bytes")
    sc = _scratch(nb.value, dev)
    _lib.check(L.uva_gutter(_p(UV), _p(F), _p(labels), m, res, int(radius), _p(img), _p(sc), nb.value, _p(out),
                            _stream(dev)), "uva_gutter")
    return img, out


def min_gutter_device(UV64, F32, labels, n_islands, res=4096, radius=64):
    """Gap between islands on device-resident FP64 UVs, int32 faces and
    labels (engine/metrics.py:348-373). Exact: the radius grows until the
    minimum is certified."""
    ntex = res * res
    r = int(radius)
    while True:
        _, out = _gutter_raw(UV64, F32, labels, res, r)
        g, filled, touch, _ = out.cpu().numpy().tolist()
        if filled == 0 or filled == ntex:
            return float("nan")
        if touch:
            return 0.0
        if g <= r or r >= 2 * res:
            break
        r = min(r * 4, 2 * res)
    if g >= 1e300:
        g = np.inf
    return max(g - 1.0, 0.0)


def min_gutter(uv, faces, islands, res=4096):
    """Smallest texel gap between two different islands (engine/metrics.py:348-373).
    Returns (gap, label image)."""
    dev = require_cuda()
    UV = torch.from_numpy(np.ascontiguousarray(uv, np.float64)).to(dev)
    F = torch.from_numpy(np.ascontiguousarray(faces, np.int32).reshape(-1, 3)).to(dev)
    lab = torch.from_numpy(np.ascontiguousarray(islands, np.int32)).to(dev)
    g = min_gutter_device(UV, F, lab, int(lab.max().item()) + 1 if len(lab) else 0, int(res))
    img, _ = _gutter_raw(UV, F, lab, int(res), 1)
    return g, to_host(img)
