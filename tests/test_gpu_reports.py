"""The report and bookkeeping drop-ins against the reference's own outputs
(tests/golden/golden_reports.npz, written by make_golden_reports.py):

* metrics.seam_report / preservation_report / full_report, with the
  in_v / in_f inputs the ComfyUI node passes (nodes.py:222, :294);
* validate.validate_uvs' preservation branch (engine/validate.py:191-199):
  exact, moved, NaN and +-0.0 corners, mismatched colours, a dropped face;
* param.boundary_edges_oriented / boundary_loops / cot_laplacian / tutte;
* gpu.unique_edges / sym_csr / csr32 / spmm and Batch._edges / Batch.L.

Tolerances: counts, masks, index arrays and booleans exact; summed lengths,
areas and distortion means 1e-9 relative (summation order differs), island
area fractions 1e-6 (the reference sums float32 cross products); FP32
products 1e-5;
p95 quantiles 1e-4 (the stated bound); Tutte UVs 1e-9 of the extent
(iterative FP64 solve to 1e-12 against the reference's LU).
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INT_KEYS = {"islands", "seam_edges", "open_boundary_edges", "nonmanifold_edge_groups", "triangles",
            "collapsed_uv_triangles", "flipped_triangles", "mirrored_islands", "islands_for_90pct_area",
            "tiny_islands_lt_0.01pct", "raster_res", "overlap_texels", "non_finite_uv", "uv_outside_unit_square",
            "degenerate_uv_triangles", "sub_float32_slivers", "overlapping_triangles_exact", "float32_contacts",
            "islands_with_overlap", "min_gutter_texels"}


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_reports.npz"))


def rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if a.size else 0.0


def check_report(got, keys, vals, what):
    ref = dict(zip(keys.tolist(), vals.tolist()))
    for k, v in ref.items():
        assert k in got, (what, k)
        x = float(got[k])
        if k in INT_KEYS or isinstance(got[k], (bool, np.bool_)):
            assert x == v, (what, k, x, v)
        elif k.endswith("_p95"):
            assert rel(x, v) <= 1e-4, (what, k, x, v)
        elif k == "largest_island_area_frac":
            # the reference sums float32 cross products of float32 positions
            assert rel(x, v) <= 1e-6, (what, k, x, v)
        else:
            assert rel(x, v) <= 1e-9 or abs(x - v) < 1e-12, (what, k, x, v)


# ------------------------------------------------------------------ param topology
@pytest.mark.parametrize("name", ["disk", "grid", "annulus", "bowtie", "dups"])
def test_boundary_edges_and_loops(g, cuda, name):
    from ultimate_uv_artist_b200.engine import param as Pm
    T = g[f"t_{name}_T"]
    bi, bj = Pm.boundary_edges_oriented(T)
    assert np.array_equal(bi, g[f"t_{name}_bi"]) and np.array_equal(bj, g[f"t_{name}_bj"])
    loops = Pm.boundary_loops(T)
    assert [len(x) for x in loops] == g[f"t_{name}_loop_len"].tolist()
    flat = np.concatenate(loops) if loops else np.zeros(0, np.int64)
    assert np.array_equal(flat, g[f"t_{name}_loops"])


def test_cot_laplacian_and_tutte(g, cuda):
    from ultimate_uv_artist_b200.engine import param as Pm
    Lc = Pm.cot_laplacian(len(g["l_P"]), g["l_T"], g["l_cots"])
    D = Lc.toarray()
    assert np.max(np.abs(D - g["l_dense"])) <= 1e-12 * np.max(np.abs(g["l_dense"]))
    for P, T, key in ((g["u_hP"], g["u_hT"], "u_tutte_hemi"), (g["u_P"], g["u_T"], "u_tutte_disk")):
        U = Pm.tutte(P, T)
        ref = g[key]
        ext = float(np.ptp(ref, 0).max())
        assert np.max(np.abs(U - ref)) <= 1e-9 * ext, key


# ------------------------------------------------------------------ gpu helpers
def test_unique_edges_and_sym_csr(g, cuda):
    from ultimate_uv_artist_b200.engine import gpu as G
    T = torch.from_numpy(g["g_T"]).to(cuda)
    n = int(g["g_n"])
    ea, eb, inv, cnt = G.unique_edges(T, n)
    for a, k in ((ea, "g_ea"), (eb, "g_eb"), (inv, "g_inv"), (cnt, "g_cnt")):
        assert a.is_cuda and np.array_equal(a.cpu().numpy(), g[k]), k
    # host tensors come back on the host
    out = G.unique_edges(torch.from_numpy(g["g_T"]), n)
    assert not out[0].is_cuda and np.array_equal(out[2].numpy(), g["g_inv"])
    keep = ea != eb
    S = G.sym_csr(n, ea[keep], eb[keep], torch.from_numpy(g["g_off"]).to(cuda), torch.from_numpy(g["g_diag"]).to(cuda))
    assert np.array_equal(S.crow_indices().cpu().numpy(), g["g_crow"])
    assert np.array_equal(S.col_indices().cpu().numpy(), g["g_col"])
    assert np.array_equal(S.values().cpu().numpy(), g["g_val"])
    X = torch.from_numpy(g["g_X"]).to(cuda)
    Y = G.spmm(S, X)
    assert rel(Y.cpu().numpy(), g["g_spmm64"]) <= 1e-12 or np.max(np.abs(Y.cpu().numpy() - g["g_spmm64"])) < 1e-13
    S32 = torch.sparse_csr_tensor(S.crow_indices(), S.col_indices(), S.values().float(), S.shape)
    assert np.allclose(G.spmm(S32, X.float()).cpu().numpy(), g["g_spmm32"], rtol=1e-5, atol=1e-5)
    assert np.allclose(G.spmm(S32, X[:, 0].float().contiguous()).cpu().numpy(), g["g_spmv32"], rtol=1e-5, atol=1e-5)
    # csr32 of a COO matrix: the same int32 layout
    coo = torch.sparse_coo_tensor(torch.from_numpy(g["g_coo_idx"]), torch.from_numpy(g["g_coo_val"]), (n, n)).to(cuda)
    C32 = G.csr32(coo)
    assert C32.crow_indices().dtype == torch.int32 and C32.col_indices().dtype == torch.int32
    assert np.array_equal(C32.crow_indices().cpu().numpy(), g["g_crow"])
    assert np.array_equal(C32.col_indices().cpu().numpy(), g["g_col"])
    with pytest.raises(IndexError):
        G.unique_edges(T, 3)


def test_batch_edges_and_laplacian(golden, cuda):
    """Batch._edges from the plan's numbering equals unique_edges of the
    batch triangles; Batch.L (float64 batch) equals the FP64 oracle's
    Laplacian, which is pinned to the reference's gpu.Batch."""
    from oracle import arap as O
    from ultimate_uv_artist_b200.engine import gpu as G
    items = [(golden[f"b_P{k}"], golden[f"b_T{k}"], golden[f"b_U{k}"]) for k in range(int(golden["b_nc"]))]
    b = G.Batch(items, dtype=torch.float64)
    ea, eb, cnt = b._edges
    ua, ub, _, uc = G.unique_edges(b.T, b.n)
    for x, y in ((ea, ua), (eb, ub), (cnt, uc)):
        assert torch.equal(x, y)
    L = b.L.to_dense().cpu().numpy()
    ref = O.BatchRef(items)
    Lr = ref.L.toarray()
    assert np.max(np.abs(L - Lr)) <= 1e-12 * np.max(np.abs(Lr))
    # no degenerate triangles here: the Jacobi diagonal is 1 / diag(L)
    assert np.allclose(b.dinv.cpu().numpy(), 1.0 / np.diag(Lr), rtol=1e-12)
    x = torch.randn(b.n, 2, dtype=torch.float64, device=cuda)
    assert torch.allclose(G.spmm(b.L, x), torch.from_numpy(Lr).to(cuda) @ x, rtol=1e-12, atol=1e-12)


# ------------------------------------------------------------------ reports
@pytest.mark.parametrize("name", ["plane", "box", "fin"])
def test_seam_and_full_report(g, cuda, name):
    from ultimate_uv_artist_b200.engine import metrics as M
    ov, of, ouv = g[f"r_{name}_ov"], g[f"r_{name}_of"], g[f"r_{name}_ouv"]
    check_report(M.seam_report(ov, of, ouv), g[f"r_{name}_seam_keys"], g[f"r_{name}_seam_vals"], "seam")
    check_report(M.seam_report(ov, of, ouv, weld_keys=g[f"r_{name}_wk"]), g[f"r_{name}_seamw_keys"],
                 g[f"r_{name}_seamw_vals"], "seam weld_keys")
    rep, isl = M.full_report(ov, of, ouv, raster_res=256, in_v=g[f"r_{name}_V"], in_f=g[f"r_{name}_F"])
    check_report(rep, g[f"r_{name}_full_keys"], g[f"r_{name}_full_vals"], "full")
    from oracle import validate as OV
    assert OV.same_partition(isl, g[f"r_{name}_isl"])


PRES = ["exact", "moved", "nan", "signed_zero", "colors", "missing", "dropped", "dtype"]


@pytest.mark.parametrize("name", PRES)
def test_preservation_report(g, cuda, name):
    from ultimate_uv_artist_b200.engine import metrics as M

    def attrs(side):
        names = g[f"p_{name}_{side}_names"].tolist()
        if not names:
            return None
        none = set(g[f"p_{name}_{side}_none"].tolist())
        return {k: (None if k in none else g[f"p_{name}_{side}_{k}"]) for k in names}

    ia, oa = attrs("ia"), attrs("oa")
    got = M.preservation_report(g[f"p_{name}_in_v"], g[f"p_{name}_in_f"], g[f"p_{name}_out_v"], g[f"p_{name}_out_f"],
                                ia, oa)
    ref = dict(zip(g[f"p_{name}_keys"].tolist(), g[f"p_{name}_vals"].tolist()))
    assert {k: bool(v) for k, v in got.items()} == ref


VAL = ["exact", "moved", "nan", "signed_zero", "colors", "dropped"]


@pytest.mark.parametrize("name", VAL)
def test_validate_preservation_branch(g, cuda, name):
    from ultimate_uv_artist_b200.engine import validate as Vd
    kw = {}
    for k in ("in_v", "in_f", "in_normals", "out_normals", "in_colors", "out_colors"):
        key = f"vv_{name}_{k}"
        if key in g:
            kw[k] = g[key]
    rep, prob = Vd.validate_uvs(g[f"vv_{name}_v"], g["vv_of"], g["vv_ouv"], atlas=512, padding=4, **kw)
    ref = dict(zip(g[f"vv_{name}_keys"].tolist(), g[f"vv_{name}_vals"].tolist()))
    assert set(ref) == {k for k, v in rep.items() if isinstance(v, (int, float, bool, np.integer, np.floating))}
    for k, v in ref.items():
        assert float(rep[k]) == v, (k, rep[k], v)
    assert np.array_equal(prob, g[f"vv_{name}_prob"])
