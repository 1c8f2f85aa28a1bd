"""ctypes binding of the C ABI in include/uva_b200.h (libuva_b200.so).

The library is required: there is no CPU fallback. Importing this module
loads the in-tree ``libuva_b200.so`` (building it with nvcc if it is missing
and a compiler is present) and raises ``RuntimeError`` otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuva_b200.so")

UVA_OK = 0
UVA_E_ARG = -1
UVA_E_CUDA = -2
UVA_E_NOBOUNDARY = -3
UVA_E_TOOBIG = -4
UVA_E_NODEVICE = -5
SEM_BATCH = 0
SEM_PARAM = 1
ST_MAXITER = 1
ST_NONFINITE = 2
ST_ENERGYSTOP = 4
ST_NOBOUNDARY = 8
ST_BADCLASS = 16

PLAN_NSIZES = 9
STEP_SETUP, STEP_LSCM, STEP_ARAP = 1, 2, 4
CLASS_BIG, CLASS_MID, CLASS_SMALL = 8192, 2048, 256
(PLAN_NC, PLAN_N, PLAN_T, PLAN_E, PLAN_NSLICES, PLAN_NSLOTS, PLAN_NBVERTS, PLAN_MAXROWS, PLAN_NCOARSE) = range(9)

vp = C.c_void_p
i32 = C.c_int32


class IslandStatus(C.Structure):
    _fields_ = [("cg_iters", i32), ("refinements", i32), ("outer_iters", i32), ("flags", i32),
                ("resid", C.c_double * 2), ("energy", C.c_double), ("step", C.c_double),
                ("t_begin", C.c_int64), ("t_end", C.c_int64), ("sm", i32), ("team", i32)]


class BatchDesc(C.Structure):
    """Mirror of ``uva_batch`` (field order and types must match the header)."""
    _fields_ = [("nc", i32), ("n", i32), ("t", i32), ("E", i32), ("nslices", i32), ("nslots", i32),
                ("semantics", i32), ("maxrows", i32),
                ("vofs", vp), ("tofs", vp), ("sofs", vp), ("tri4", vp), ("tri_edge", vp),
                ("slice_ptr", vp), ("slot_col", vp), ("slot_edge", vp), ("slot_c", vp),
                ("vt_ptr", vp), ("vt", vp), ("vflags", vp), ("bofs", vp), ("bverts", vp), ("order", vp),
                ("row_vert", vp), ("vert_row", vp), ("agg_rows", vp), ("cofs", vp),
                ("coarse_a", vp), ("coarse_l", vp), ("coarse_work", vp), ("cpart", vp),
                ("class_ofs", i32 * 5),
                ("P", vp), ("frame", vp), ("wtri", vp), ("tscale", vp), ("wedge", vp), ("slot_cw", vp),
                ("wdiag", vp), ("dinv", vp), ("pins", vp), ("wpin", vp), ("U", vp),
                ("x64", vp), ("b64", vp), ("rc", vp), ("r32", vp), ("d32", vp), ("p32", vp), ("q32", vp),
                ("status", vp), ("work", vp), ("hist", vp)]


class DPlanDesc(C.Structure):
    """Mirror of ``uva_dplan``."""
    _fields_ = [("nc", i32), ("n", i32), ("t", i32), ("nslices", i32),
                ("vofs", vp), ("tofs", vp), ("T", vp), ("agg_rows", vp), ("sofs", vp),
                ("tri4", vp), ("tri_edge", vp), ("slice_ptr", vp), ("vt_ptr", vp), ("vt", vp),
                ("vflags", vp), ("bofs", vp), ("bverts", vp), ("row_vert", vp), ("vert_row", vp),
                ("sizes", vp), ("scratch", vp), ("scratch_bytes", C.c_int64)]


class SolveParams(C.Structure):
    _fields_ = [("iters", i32), ("line_search", i32), ("tol", C.c_double), ("energy_tol", C.c_double),
                ("inner_eta", C.c_double), ("max_inner", i32), ("max_refine", i32), ("threads", i32),
                ("rev_ctas", i32), ("fold_step", i32)]


class SegDesc(C.Structure):
    """Mirror of ``uva_seg_desc``."""
    _fields_ = [("nc", i32), ("nseg", i32), ("n", i32), ("mode", i32), ("max_report", i32), ("reserved", i32),
                ("U", vp), ("vofs", vp), ("seg_ofs", vp), ("seg", vp), ("out", vp), ("scratch", vp),
                ("scratch_bytes", C.c_int64)]


SEG_COUNT, SEG_ANY, SEG_ANY_ALL, SEG_FIRST = 0, 1, 2, 3

_SIGS = {
    "uva_plan_create": [vp, vp, vp, i32, i32, vp],
    "uva_plan_create_charts": [vp, vp, vp, vp, i32, i32, vp],
    "uva_plan_sizes": [vp, vp],
    "uva_plan_export": [vp] * 13,
    "uva_plan_export_range": [vp, i32, i32] + [vp] * 12,
    "uva_plan_island_offsets": [vp, vp],
    "uva_plan_export_rows": [vp] * 5,
    "uva_plan_destroy": [vp],
    "uva_concat_charts": [i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32],
    "uva_batch_setup": [vp, vp],
    "uva_lscm": [vp, vp, vp],
    "uva_arap": [vp, vp, vp],
    "uva_arap_noalloc": [vp, vp, vp],
    "uva_slim": [vp, vp, vp, vp],
    "uva_slim_scratch_bytes": [vp, vp],
    "uva_step_graph_create": [vp, i32, vp, vp, vp],
    "uva_graph_launch": [vp, vp],
    "uva_graph_destroy": [vp],
    "uva_orient_positive": [vp, vp],
    "uva_repair_flips": [vp, i32, vp],
    "uva_repair_flips_serial": [vp, i32, vp],
    "uva_flips_per_chart": [vp, vp, vp],
    "uva_signed_area": [vp, vp, vp, vp],
    "uva_jacobians": [vp, vp, vp, vp],
    "uva_shrink": [vp, vp, vp, i32, C.c_float, C.c_float, vp],
    "uva_seg_scratch_bytes": [i32, i32, vp],
    "uva_csr_pcg_blocks": [i32, vp, i32, vp, vp, vp, vp, vp, C.c_double, i32, vp, vp, vp],
    "uva_hier_boundary_corners": [vp, vp, C.c_int64, vp, vp, vp, vp, C.c_int64, C.c_int64, vp, vp, vp, vp],
    "uva_hier_lscm_scratch_bytes": [C.c_int64, C.c_int64, C.c_int64, i32, vp],
    "uva_hier_lscm": [vp, C.c_int64, vp, C.c_int64, vp, vp, vp, C.c_int64, C.c_int64, i32, vp, vp, vp, C.c_int64,
                      C.c_double, i32, vp, C.c_int64, vp, vp, vp],
    "uva_overlap_raster": [vp, vp, i32, i32, vp, vp, vp, C.c_int64, vp],
    "uva_gutter_scratch_bytes": [i32, C.c_int64, vp],
    "uva_boundary_hits": [vp, vp],
    "uva_batch_boundary_scratch_bytes": [vp, vp],
    "uva_batch_boundary": [vp, vp, vp, vp, C.c_int64, vp],
    "uva_unique_edges_scratch_bytes": [C.c_int64, C.c_int64, vp],
    "uva_unique_edges": [vp, C.c_int64, C.c_int64, vp, vp, vp, vp, vp, vp, C.c_int64, vp],
    "uva_sym_csr_scratch_bytes": [C.c_int64, vp],
    "uva_sym_csr": [C.c_int64, C.c_int64, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, C.c_int64, vp],
    "uva_csr_spmm": [i32, i32, C.c_int64, vp, vp, vp, vp, vp, i32, vp],
    "uva_boundary_mask_scratch_bytes": [C.c_int64, vp],
    "uva_boundary_mask": [vp, C.c_int64, vp, vp, vp, C.c_int64, vp],
    "uva_batch_edges": [vp, vp, vp, vp, vp],
    "uva_seam_report_scratch_bytes": [C.c_int64, C.c_int64, vp],
    "uva_seam_report": [vp, C.c_int64, vp, C.c_int64, vp, vp, vp, vp, vp, C.c_int64, vp],
    "uva_corners_equal": [vp, i32, C.c_int64, vp, vp, i32, C.c_int64, vp, C.c_int64, i32, vp, vp],
    "uva_segment_sum": [vp, C.c_int64, vp, C.c_int64, i32, vp, vp, vp],
    "uva_validate_finish": [vp, vp],
    "uva_concat_tris32": [i32, vp, vp, vp, vp, i32],
    "uva_concat_rows32": [i32, vp, vp, i32, vp, i32],
    "uva_dplan_scratch_bytes": [C.c_int64, C.c_int64, C.c_int64, vp],
    "uva_dplan_build": [vp, vp],
    "uva_dplan_slots": [vp, vp, vp, vp, vp],
    "uva_pack_scratch_bytes": [C.c_int64, C.c_int64, C.c_int64, i32, i32, vp],
    "uva_pack_masks": [vp, vp],
    "uva_pack_place": [vp, i32, vp],
    "uva_pack_place_pages": [vp, i32, i32, vp],
    "uva_pack_uv": [vp, i32, i32, vp, C.c_int64, C.c_double, vp, vp, vp],
    "uva_last_error": [],
    "uva_version": [],
}

_lock = threading.Lock()
_lib = None


def _load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            try:
                from . import build as _build
                _build.build()
            except Exception as exc:  # noqa: BLE001 - re-raised with context
                raise RuntimeError(f"uva_b200: {LIB_PATH} is missing and could not be built: {exc}") from exc
        lib = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = i32
        lib.uva_last_error.restype = C.c_char_p
        lib.uva_plan_destroy.restype = None
        _lib = lib
        return lib


def lib():
    return _load()


_pyhost = None


def pyhost():
    """The batch constructor's host helper (libuva_pyhost.so, called with the
    GIL held), or None when it is missing: the constructor then reads the
    charts in Python."""
    global _pyhost
    if _pyhost is None:
        path = os.path.join(HERE, "libuva_pyhost.so")
        handle = False
        if os.path.exists(path):
            try:
                h = C.PyDLL(path)
                h.uva_py_charts.argtypes = [C.py_object, i32] + [vp] * 9
                h.uva_py_charts.restype = C.c_int64
                handle = h
            except OSError:
                handle = False
        _pyhost = handle
    return _pyhost or None


def exported_symbols():
    """Names this binding expects the library to export."""
    return sorted(_SIGS)


def check(status, what=""):
    """Raise on a non-zero status, with the library's thread-local message."""
    if status == UVA_OK:
        return
    msg = lib().uva_last_error().decode(errors="replace")
    if status == UVA_E_NOBOUNDARY:
        raise ValueError(msg or "chart has no boundary (closed surface): needs a cut")
    if status == UVA_E_ARG:
        raise ValueError(f"{what}: {msg}")
    raise RuntimeError(f"{what}: uva_b200 status {status}: {msg}")


def ptr(t):
    """Raw device/host address of a torch tensor or numpy array (None -> 0)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


def stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)
