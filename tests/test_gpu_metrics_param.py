"""GPU metrics (engine/metrics.py) and per-chart param helpers
(engine/param.py) against the reference's own outputs (golden fixtures).

Tolerances: FP64 geometry 1e-9 relative; p95 quantiles 1e-4 relative (the
the stated bound on p95 anisotropy); rasters, counts and the serial flip
repair bit-exact."""
import numpy as np
import pytest

from oracle import arap as O
from oracle import validate as OV

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if a.size else 0.0


def test_triangle_jacobians(golden, cuda):
    from ultimate_uv_artist_b200.engine import metrics as M
    V, F, UV = golden["v_V"].astype(np.float64), golden["v_F"], golden["v_UV"].astype(np.float64)
    s1, s2, sa, A3, good = M.triangle_jacobians(V[F], UV[F])
    assert np.allclose(s1, golden["v_s1"], rtol=1e-9, atol=1e-12)
    assert np.allclose(s2, golden["v_s2"], rtol=1e-7, atol=1e-9)
    assert np.allclose(sa, golden["v_sa"], rtol=1e-12, atol=1e-18)
    assert np.allclose(A3, golden["v_A3"], rtol=1e-12)
    assert np.array_equal(good, golden["v_good"])


def test_distortion_report(golden, cuda):
    from ultimate_uv_artist_b200.engine import metrics as M
    ref = dict(zip(golden["v_dist_keys"].tolist(), golden["v_dist_vals"].tolist()))
    got = M.distortion_report(golden["v_V"], golden["v_F"], golden["v_UV"].astype(np.float64), golden["v_isl"])
    for k, v in ref.items():
        if k.endswith("_p95"):
            assert rel(got[k], v) <= 1e-4, (k, got[k], v)
        elif k in ("triangles", "collapsed_uv_triangles", "flipped_triangles", "mirrored_islands"):
            assert got[k] == int(v), (k, got[k], v)
        else:
            assert rel(got[k], v) <= 1e-9 or abs(got[k] - v) < 1e-12, (k, got[k], v)


def test_rasters_and_islands(golden, cuda):
    from ultimate_uv_artist_b200.engine import metrics as M
    U64 = golden["v_UV"].astype(np.float32).astype(np.float64)
    counts, occ, ov = M.raster_coverage(U64, golden["v_F"], 256)
    assert np.array_equal(counts, golden["v_counts"])
    lab, n = M.uv_islands(golden["v_F"], len(golden["v_V"]), U64, golden["v_V"])
    assert n == int(golden["v_nisl"]) and OV.same_partition(lab, golden["v_isl"])
    img = np.full((512, 512), -1, np.int32)
    M._raster_labels(U64, golden["v_F"], golden["v_isl"], 512, img)
    assert np.array_equal(img, golden["v_img"])
    Uw = golden["w_UV"].astype(np.float32).astype(np.float64)
    g, _ = M.min_gutter(Uw, golden["w_F"], golden["w_isl"], 512)
    assert g == float(golden["w_gutter"])


def test_param_helpers(golden, cuda):
    from ultimate_uv_artist_b200.engine import param as Pm
    P, T = golden["p_P"], golden["p_T"]
    X, area = Pm.local_frames(P, T)
    assert np.allclose(X, golden["p_X"], rtol=1e-12, atol=1e-14) and np.allclose(area, golden["p_area"], rtol=1e-12)
    cots = Pm.cot_weights(golden["p_X"])
    assert np.allclose(cots, golden["p_cots"], rtol=1e-10, atol=1e-12)
    R, _ = Pm._arap_rotations(golden["p_U0"], T, golden["p_X"], golden["p_cots"], 0, False)
    assert np.allclose(R, golden["p_R"], atol=1e-12)
    b = Pm._arap_rhs(len(P), T, golden["p_X"], golden["p_cots"], golden["p_R"])
    assert np.allclose(b, golden["p_b"], atol=1e-12)
    ms = Pm._max_step(golden["p_U0"], golden["p_U1"] - golden["p_U0"], T)
    assert rel(ms, golden["p_maxstep"]) < 1e-12
    assert rel(Pm._energy(golden["p_U1"], T, golden["p_X"], golden["p_area"], 0), golden["p_E0"]) < 1e-10
    assert rel(Pm._energy(golden["p_U1"], T, golden["p_X"], golden["p_area"], 1), golden["p_E1"]) < 1e-10
    sa = Pm.signed_areas(golden["p_U1"], T)
    assert np.allclose(sa, O.signed_areas(golden["p_U1"], T), rtol=1e-12, atol=1e-18)


def test_param_solvers(golden, cuda):
    from ultimate_uv_artist_b200.engine import param as Pm
    P, T = golden["p_P"], golden["p_T"]
    ext = np.ptp(golden["p_U0"], 0).max()
    U0 = Pm.lscm(P, T)
    assert np.abs(U0 - golden["p_U0"]).max() / ext < 1e-7
    U1, solver = Pm.refine(P, T, golden["p_U0"], iters=10, tol=0.0)
    assert np.abs(U1 - golden["p_U1"]).max() / ext < 1e-7
    U2, _ = Pm.refine(P, T, golden["p_U0"], iters=10, tol=1e-5, solver=solver)
    assert np.abs(U2 - golden["p_U2"]).max() / ext < 1e-7
    Ur = Pm.repair_flips(golden["p_Uf"], T, rounds=60)
    assert np.array_equal(Ur, golden["p_Ur"])
    q = Pm.chart_quality(P, T, golden["p_U1"])
    assert q["flips"] == int(golden["p_q_flips"])
    assert rel(q["aniso_p95"], golden["p_q_aniso_p95"]) <= 1e-4
    assert rel(q["area_p95"], golden["p_q_area_p95"]) <= 1e-4
    assert rel(q["stretch"], golden["p_q_stretch"]) <= 1e-9
    assert np.allclose(q["per_tri_aniso"], golden["p_q_aniso"], rtol=1e-7)
    assert np.allclose(q["per_tri_area"], golden["p_q_area"], rtol=1e-9)


def test_slim_rotations_and_refine(golden, cuda):
    """SLIM (engine/param.py:206-256 mode 1, 415-454) against the reference's
    outputs. UVs are compared after removing the mean shift: the SLIM normal
    equations fix the translation only through a 1e-12 sum(area) regulariser,
    so the reference's own translation moves with its LU round-off."""
    from ultimate_uv_artist_b200.engine import param as Pm
    P, T, U0 = golden["s_P"], golden["s_T"], golden["s_U0"]
    X, area = O.local_frames(P, T)
    R, W = Pm._arap_rotations(U0, T, X, None, 1, True)
    assert np.abs(R - golden["s_R1"]).max() < 1e-12
    assert np.abs(W - golden["s_W1"]).max() < 1e-10
    ext = np.ptp(golden["s_U5"], 0).max()
    for iters, tol, key in ((5, 0.0, "s_U5"), (20, 1e-5, "s_U20")):
        U, solver = Pm.refine(P, T, U0, iters=iters, method="slim", tol=tol)
        assert solver is None
        d = U - golden[key]
        assert np.abs(d - d.mean(0)).max() / ext < 1e-5, (key, np.abs(d - d.mean(0)).max() / ext)
        assert np.abs(d.mean(0)).max() / ext < 1e-3
    U5, _ = Pm.refine(P, T, U0, iters=5, method="slim", tol=0.0)
    assert rel(Pm._energy(U5, T, X, area, 1), golden["s_E5"]) < 1e-8
    # an inverted start is returned unchanged, as the reference does
    Uf = U0.copy()
    Uf[:, 0] *= -1.0
    Ub, _ = Pm.refine(P, T, Uf, iters=3, method="slim")
    assert np.array_equal(Ub, Uf)


def test_spd_solver_and_tutte(cuda):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import param as Pm
    P, T = synth.hemisphere_patch(seed=5, n=12)
    n = len(P)
    A = (Pm.cot_laplacian(n, T, Pm.cot_weights(Pm.local_frames(P, T)[0])) + sp.eye(n) * 1e-3).tocsc()
    rng = np.random.default_rng(0)
    b = rng.normal(size=(n, 2))
    x = Pm.SPDSolver(A).solve(b)
    assert np.allclose(x, spla.spsolve(A, b), rtol=1e-8, atol=1e-10)
    # tutte (param.py:182-202) against the same construction solved by scipy
    U = Pm.tutte(P, T)
    loop = max(Pm.boundary_loops(T), key=len)
    P64 = P.astype(np.float64)
    seg = np.linalg.norm(P64[np.roll(loop, -1)] - P64[loop], axis=1)
    tt = np.r_[0, np.cumsum(seg)[:-1]] / seg.sum() * 2 * np.pi
    Ub = np.stack([np.cos(tt), np.sin(tt)], 1) * seg.sum() / (2 * np.pi)
    I = np.concatenate([T[:, 0], T[:, 1], T[:, 2], T[:, 1], T[:, 2], T[:, 0]])
    J = np.concatenate([T[:, 1], T[:, 2], T[:, 0], T[:, 0], T[:, 1], T[:, 2]])
    Adj = sp.csr_matrix((np.ones(len(I)), (I, J)), shape=(n, n))
    Adj.data[:] = 1.0
    Lu = (sp.diags(np.asarray(Adj.sum(1)).ravel()) - Adj).tocsr()
    fixed = np.zeros(n, bool); fixed[loop] = True
    ref = np.zeros((n, 2)); ref[loop] = Ub
    ref[~fixed] = spla.spsolve(Lu[~fixed][:, ~fixed].tocsc(), -Lu[~fixed][:, fixed] @ Ub)
    assert np.allclose(U, ref, atol=1e-9)
