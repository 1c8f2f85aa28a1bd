"""CPU tests: the oracle against the reference's golden fixtures, the C ABI
(library loads, every declared symbol exported), the host topology plan, and
the synthetic generators. No GPU needed."""
import os
import re

import numpy as np
import pytest

from oracle import arap as O
from oracle import validate as OV

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# ---------------------------------------------------------------- oracle vs reference
def test_oracle_param_matches_reference(golden):
    P, T = golden["p_P"], golden["p_T"]
    X, area = O.local_frames(P, T)
    assert np.array_equal(X, golden["p_X"]) and np.array_equal(area, golden["p_area"])
    cots = O.cot_weights(X)
    assert np.array_equal(cots, golden["p_cots"])
    assert np.abs(O.lscm(P, T) - golden["p_U0"]).max() < 1e-12
    bi, _ = O.boundary_edges_oriented(T)
    assert O.far_pair(P, np.unique(bi)) == tuple(golden["p_pins"].tolist())
    R = O.arap_rotations(golden["p_U0"], T, X)
    assert np.abs(R - golden["p_R"]).max() < 1e-14
    assert np.abs(O.arap_rhs(len(P), T, X, cots, R) - golden["p_b"]).max() < 1e-13
    assert np.abs(O.refine_arap(P, T, golden["p_U0"], iters=10, tol=0.0) - golden["p_U1"]).max() < 1e-12
    assert np.abs(O.refine_arap(P, T, golden["p_U0"], iters=10, tol=1e-5) - golden["p_U2"]).max() < 1e-12
    assert O.max_step_param(golden["p_U0"], golden["p_U1"] - golden["p_U0"], T) == float(golden["p_maxstep"])
    assert abs(O.energy(golden["p_U1"], T, X, area, 0) - float(golden["p_E0"])) < 1e-12
    assert np.array_equal(O.repair_flips_param(golden["p_Uf"], T), golden["p_Ur"])


def _rel_modulo_translation(U, ref):
    """Max |U - ref| over the UV extent after removing the mean shift. The
    SLIM normal equations fix the translation only through a 1e-12 sum(area)
    regulariser (engine/param.py:426-429), so the reference's own translation
    moves by about 1e-5 of the extent with the sparse LU's round-off."""
    d = U - ref
    return float(np.abs(d - d.mean(0)).max() / np.ptp(ref, 0).max())


def test_oracle_slim_matches_reference(golden):
    P, T, U0 = golden["s_P"], golden["s_T"], golden["s_U0"]
    X, area = O.local_frames(P, T)
    R, W = O.slim_local(U0, T, X)
    assert np.abs(R - golden["s_R1"]).max() < 1e-12 and np.abs(W - golden["s_W1"]).max() < 1e-11
    U5 = O.refine_slim(P, T, U0, iters=5, tol=0.0)
    assert _rel_modulo_translation(U5, golden["s_U5"]) < 1e-12
    assert abs(O.energy(U5, T, X, area, 1) - float(golden["s_E5"])) <= 1e-12 * float(golden["s_E5"])
    U20 = O.refine_slim(P, T, U0, iters=20)
    assert _rel_modulo_translation(U20, golden["s_U20"]) < 1e-12


def test_oracle_batch_matches_reference(golden):
    nc = int(golden["b_nc"])
    items = [(golden[f"b_P{k}"], golden[f"b_T{k}"], golden[f"b_U{k}"]) for k in range(nc)]
    B = O.BatchRef(items)
    assert B.wpin == float(golden["b_wpin"])
    B.orient_positive()
    assert np.abs(B.U - golden["b_Ua"]).max() < 1e-15
    assert np.abs(B.rhs(B.U) - golden["b_rhs0"]).max() < 1e-12
    B.arap(6, True)
    assert O.uv_rel_error(B.U, golden["b_Ub"], B.offsets) < 1e-9
    B.arap(3, False)
    assert O.uv_rel_error(B.U, golden["b_Uc"], B.offsets) < 1e-9
    B.U = golden["b_Ud"].copy()
    assert np.array_equal(B.flips_per_chart(), golden["b_flips"])
    B.repair_flips(40)
    assert np.abs(B.U - golden["b_Ue"]).max() < 1e-12


@pytest.mark.parametrize("prefix", ["v", "w"])
def test_oracle_validation_matches_reference(golden, prefix):
    V, F, UV = golden[f"{prefix}_V"], golden[f"{prefix}_F"], golden[f"{prefix}_UV"]
    rep, prob, ex = OV.validate_uvs(V, F, UV, atlas=512, padding=4)
    ref = dict(zip(golden[f"{prefix}_rep_keys"].tolist(), golden[f"{prefix}_rep_vals"].tolist()))
    for k, v in ref.items():
        assert float(rep[k]) == v, (k, rep[k], v)
    assert np.array_equal(prob, golden[f"{prefix}_problems"])
    assert OV.same_partition(ex["islands"], golden[f"{prefix}_isl"])
    if prefix == "v":
        assert np.array_equal(ex["ov"], golden["v_ov"]) and np.array_equal(ex["ov_strict"], golden["v_ovs"])
        U64 = UV.astype(np.float32).astype(np.float64)
        assert np.array_equal(OV.raster_labels(U64, F, golden["v_isl"], 512), golden["v_img"])
        assert np.array_equal(OV.raster_counts(U64, F, 256), golden["v_counts"])
        assert np.array_equal(OV.chart_overlaps(golden["v_cU"], golden["v_cF"]), golden["v_cov"])


def test_numpy_predicates_agree_with_c_loops(golden):
    """The vectorised numpy predicates and the C restatement of the serial
    loops give the same flags (two independent restatements)."""
    V, F, UV = golden["v_V"], golden["v_F"], golden["v_UV"]
    U = UV.astype(np.float32).astype(np.float64)
    skip = np.zeros(len(F), bool)
    for strict in (False, True):
        a, _ = OV.overlaps(U, F, skip, 0.0 if strict else 1e-6, strict=strict)
        b, _ = OV.overlaps_c(U, F, skip, 64, 0.0 if strict else 1e-6, strict=strict)
        assert np.array_equal(a, b)
    lab = golden["v_isl"]
    assert np.array_equal(OV.raster_labels_numpy(U, F, lab, 128), OV.raster_labels(U, F, lab, 128))


# ---------------------------------------------------------------- C ABI
def _declared_functions():
    src = open(os.path.join(ROOT, "include", "uva_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(uva_[a-z_0-9]+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from ultimate_uv_artist_b200 import _lib
    L = _lib.lib()
    names = _declared_functions()
    assert len(names) >= 30, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.uva_version() >= 1


def test_plan_matches_numpy_topology():
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.device import Plan, concat_charts
    rng = np.random.default_rng(1)
    isl = [synth.disk_patch(rng, t) for t in (20, 150, 900)] + [synth.hemisphere_patch(seed=3, n=9)]
    P, T, _, vofs, tofs = concat_charts([(p, t) for p, t in isl], with_uv=False)
    pl = Plan(T, vofs, tofs)
    assert pl.n == len(P) and pl.t == len(T)
    for i in range(pl.nc):
        Ti = T[tofs[i]:tofs[i + 1]]
        n = vofs[i + 1] - vofs[i]
        a = np.r_[Ti[:, 1], Ti[:, 2], Ti[:, 0]]
        b = np.r_[Ti[:, 2], Ti[:, 0], Ti[:, 1]]
        key = np.unique(np.minimum(a, b) * n + np.maximum(a, b))
        ea, eb = key // n, key % n
        rv, vr = pl.row_vert[vofs[i]:vofs[i + 1]], pl.vert_row[vofs[i]:vofs[i + 1]]
        assert np.array_equal(np.sort(rv), np.arange(n)) and np.array_equal(rv[vr], np.arange(n))
        if n > 256:   # aggregates of agg_rows consecutive rows, at most 256 of them
            m = -(-n // pl.agg_rows[i])
            assert pl.agg_rows[i] % 64 == 0 and m <= 256 and pl.cofs[i + 1] - pl.cofs[i] == m * m
        else:
            assert pl.agg_rows[i] == 0 and pl.cofs[i + 1] == pl.cofs[i] and np.array_equal(rv, np.arange(n))
        for v in range(n):
            row = vr[v]
            s = pl.sofs[i] + row // 32
            w = (pl.slice_ptr[s + 1] - pl.slice_ptr[s]) // 32
            assert w % 4 == 0
            q = pl.slice_ptr[s] + row % 32 + 32 * np.arange(w)
            cols = [int(rv[c]) for c, e in zip(pl.slot_col[q], pl.slot_edge[q]) if e >= 0]
            assert cols == sorted(set(eb[ea == v].tolist()) | set(ea[eb == v].tolist()))
        bi, bj = O.boundary_edges_oriented(Ti)
        assert np.array_equal(np.unique(bi), pl.bverts[pl.bofs[i]:pl.bofs[i + 1]])
    # island work order: classes by vertex count, each class largest first
    nv = np.diff(vofs)[pl.order]
    assert np.all(np.diff(pl.class_ofs) >= 0) and pl.class_ofs[-1] == pl.nc


def test_plan_rejects_bad_indices():
    from ultimate_uv_artist_b200.device import Plan
    T = np.array([[0, 1, 5]])
    with pytest.raises(ValueError):
        Plan(T, [0, 3], [0, 1])


def test_product_path_requires_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from ultimate_uv_artist_b200.engine import gpu
    with pytest.raises(RuntimeError):
        gpu.Batch([(np.zeros((3, 3)), np.array([[0, 1, 2]]), np.zeros((3, 2)))])


# ---------------------------------------------------------------- generators
def test_validation_atlas_faults():
    from ultimate_uv_artist_b200 import synth
    V, F, UV, info = synth.validation_atlas(seed=31, islands=60, tris_per_island=50, atlas=512, padding=4,
                                            overlap_rate=2e-3, fold_rate=2e-3, mirrored=2, outside=5)
    assert len(info["mirrored"]) == 2 and len(info["outside"]) == 5
    assert ((UV < 0) | (UV > 1)).any(1).sum() == 5


def test_uneven_islands_sizes():
    from ultimate_uv_artist_b200 import synth
    isl = synth.uneven_islands(seed=7, count=50)
    t = np.array([len(T) for _, T in isl])
    assert t.min() >= 8 and t.max() <= 20000


def test_concat_charts_matches_numpy():
    """uva_concat_charts widens and places every chart like numpy's
    concatenation (gpu.Batch.__init__'s copies), for mixed input dtypes."""
    from ultimate_uv_artist_b200.device import concat_charts
    rng = np.random.default_rng(4)
    charts = []
    for k in range(40):
        nv, nt = int(rng.integers(3, 60)), int(rng.integers(1, 90))
        P = rng.standard_normal((nv, 3)).astype(np.float32 if k % 2 else np.float64)
        T = rng.integers(0, nv, (nt, 3)).astype(np.int32 if k % 3 else np.int64)
        U = None if k % 4 == 0 else rng.standard_normal((nv, 2)).astype(np.float32 if k % 5 else np.float64)
        charts.append((P, T, U))
    charts.append((np.zeros((0, 3)), np.zeros((0, 3), np.int64), None))   # empty chart
    P, T, U, vofs, tofs = concat_charts(charts)
    assert np.array_equal(P, np.concatenate([c[0].astype(np.float64) for c in charts]))
    assert np.array_equal(T, np.concatenate([c[1].astype(np.int64) for c in charts]))
    assert np.array_equal(U, np.concatenate([np.zeros((len(c[0]), 2)) if c[2] is None else c[2].astype(np.float64)
                                             for c in charts]))
    assert np.array_equal(np.diff(vofs), [len(c[0]) for c in charts])
    with pytest.raises(ValueError):
        concat_charts([(np.zeros((4, 3)), np.zeros((1, 3), np.int64), np.zeros((3, 2)))])
    assert concat_charts([c[:2] + (None,) for c in charts])[2] is None   # no UVs: nothing to upload


def test_plan_from_chart_arrays_matches_concatenated():
    """uva_plan_create_charts (per-chart int32 / int64 triangle arrays, no
    concatenation) builds the same plan as uva_plan_create."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.device import Plan, concat_charts
    isl = synth.uneven_islands(seed=61, count=30, tmin=20, tmax=3000)
    charts = [(p, t.astype(np.int32) if k % 2 else t, None) for k, (p, t) in enumerate(isl)]
    P, T, _, vofs, tofs = concat_charts(charts)
    P2, Tc, _, vofs2, tofs2 = concat_charts(charts, with_t=False)
    assert np.array_equal(P, P2) and np.array_equal(vofs, vofs2) and np.array_equal(tofs, tofs2)
    a = Plan(T, vofs, tofs)
    b = Plan(None, vofs2, tofs2, chart_tris=Tc[:2])
    for k in ("tri4", "tri_edge", "sofs", "slice_ptr", "slot_col", "slot_edge", "slot_c", "vt_ptr", "vt", "vflags",
              "bofs", "bverts", "order", "row_vert", "vert_row", "agg_rows", "cofs"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    bad = [(p, t.copy(), None) for p, t, _ in charts]
    bad[3][1][0, 0] = len(bad[3][0])                   # a vertex id outside its chart
    _, Tb, _, vb, tb = concat_charts(bad, with_t=False)
    with pytest.raises(ValueError):
        Plan(None, vb, tb, chart_tris=Tb[:2])


def test_plan_range_export_matches_full_export():
    """uva_plan_export_range over consecutive island ranges writes the same
    arrays as one uva_plan_export (the ranges a device copy pipeline uses)."""
    import ctypes as C
    from ultimate_uv_artist_b200 import _lib, synth
    from ultimate_uv_artist_b200.device import Plan, concat_charts
    isl = synth.uneven_islands(seed=62, count=25, tmin=20, tmax=3000)
    P, T, _, vofs, tofs = concat_charts([(p, t) for p, t in isl], with_uv=False)
    full = Plan(T, vofs, tofs)
    L = _lib.lib()
    Tl = np.ascontiguousarray(T, np.int64)
    v64, t64 = np.ascontiguousarray(vofs, np.int64), np.ascontiguousarray(tofs, np.int64)
    h = C.c_void_p()
    _lib.check(L.uva_plan_create(_lib.ptr(Tl), _lib.ptr(v64), _lib.ptr(t64), len(vofs) - 1, 0, C.byref(h)), "create")
    out = {k: np.full_like(getattr(full, k), 77) for k in Plan.EXPORTED}
    args = [_lib.ptr(out[k]) for k in Plan.EXPORTED]
    for i0, i1 in ((0, 7), (7, 8), (8, 20), (20, 25)):
        _lib.check(L.uva_plan_export_range(h, i0, i1, *args), "export_range")
    off = np.zeros(3 * 26, np.int64)
    _lib.check(L.uva_plan_island_offsets(h, _lib.ptr(off)), "offsets")
    L.uva_plan_destroy(h)
    for k in Plan.EXPORTED:
        assert np.array_equal(out[k], getattr(full, k)), k
    assert np.array_equal(off[:26], full.sofs) and np.array_equal(off[52:], full.bofs)


def test_boundary_loop_walk_against_reference():
    """The host loop walk of param.boundary_loops on the reference's own
    boundary half-edges (golden_reports.npz): same loops, same order."""
    from ultimate_uv_artist_b200.engine.param import _trace_loops
    g = np.load(os.path.join(ROOT, "tests", "golden", "golden_reports.npz"))
    for name in ("disk", "grid", "annulus", "bowtie", "dups"):
        loops = _trace_loops(g[f"t_{name}_bi"], g[f"t_{name}_bj"])
        assert [len(x) for x in loops] == g[f"t_{name}_loop_len"].tolist(), name
        flat = np.concatenate(loops) if loops else np.zeros(0, np.int64)
        assert np.array_equal(flat, g[f"t_{name}_loops"]), name


def test_cot_laplacian_assembly_against_reference():
    """param.cot_laplacian (host scipy assembly) equals the reference's matrix."""
    from ultimate_uv_artist_b200.engine import param as Pm
    g = np.load(os.path.join(ROOT, "tests", "golden", "golden_reports.npz"))
    D = Pm.cot_laplacian(len(g["l_P"]), g["l_T"], g["l_cots"]).toarray()
    assert np.max(np.abs(D - g["l_dense"])) <= 1e-12 * np.max(np.abs(g["l_dense"]))
    I, J, W = Pm._lap_triplets(g["l_T"], g["l_cots"])
    import scipy.sparse as sp
    D2 = sp.coo_matrix((W, (I, J)), shape=D.shape).toarray()
    assert np.max(np.abs(D2 - g["l_dense"])) <= 1e-12 * np.max(np.abs(g["l_dense"]))


def test_oracle_chart_quality_against_reference(golden):
    """oracle.arap.chart_quality equals the reference's param.chart_quality
    (golden_small.npz, the refined hemisphere patch)."""
    q = O.chart_quality(golden["p_P"], golden["p_T"], golden["p_U1"])
    assert q["flips"] == int(golden["p_q_flips"])
    assert abs(q["aniso_p95"] - float(golden["p_q_aniso_p95"])) <= 1e-12 * abs(float(golden["p_q_aniso_p95"]))
    assert abs(q["area_p95"] - float(golden["p_q_area_p95"])) <= 1e-12 * abs(float(golden["p_q_area_p95"]))
    assert abs(q["stretch"] - float(golden["p_q_stretch"])) <= 1e-12 * abs(float(golden["p_q_stretch"]))
    assert np.allclose(q["per_tri_aniso"], golden["p_q_aniso"], rtol=1e-12)
    assert np.allclose(q["per_tri_area"], golden["p_q_area"], rtol=1e-12)


def test_chart_arrays_native_pass_matches_python_path(monkeypatch):
    """The native charts pass (libuva_pyhost.so) and the Python path give
    the same codes, offsets and concatenated arrays, for charts the host
    copies read as they are and for charts that need a conversion."""
    from ultimate_uv_artist_b200 import _lib
    from ultimate_uv_artist_b200.device import ChartArrays
    assert _lib.pyhost() is not None
    rng = np.random.default_rng(3)
    charts = [(rng.random((5, 3)).astype(np.float32), np.array([[0, 1, 2], [2, 3, 4]], np.int32), None),
              (rng.random((4, 3)), np.array([[0, 1, 2]], np.uint32), rng.random((4, 2)).astype(np.float32)),
              (rng.random(9).tolist(), [[0, 1, 2]], None),
              (np.asfortranarray(rng.random((3, 3))), np.array([[0, 1, 2]]), rng.random((3, 2)).astype(np.float16)),
              (rng.random((6, 3)), np.array([[0, 1, 2], [3, 4, 5]], np.int64), rng.random((6, 2)))]
    fast = ChartArrays(charts)
    Pf, Uf = fast.points()
    monkeypatch.setattr(_lib, "_pyhost", False)
    slow = ChartArrays(charts)
    Ps, Us = slow.points()
    for k in ("pdt", "tdt", "udt", "vofs", "tofs"):
        assert np.array_equal(getattr(fast, k), getattr(slow, k)), k
    assert fast.any_uv == slow.any_uv
    assert np.array_equal(Pf, Ps) and np.array_equal(Uf, Us)
    with pytest.raises(ValueError):
        ChartArrays([(np.zeros((4, 3)), np.zeros((1, 3), np.int64), np.zeros((3, 2)))])
