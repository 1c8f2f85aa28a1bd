"""GPU parity of the batched LSCM / ARAP path against the reference's own
outputs (golden fixtures) and the FP64 oracle.

Tolerances: UVs within 1e-5 relative to each chart's UV
extent; p95 anisotropy within 1e-4; global steps at 1e-6 relative residual
per column, checked in FP64.
"""
import numpy as np
import pytest
import torch

from oracle import arap as O

pytestmark = pytest.mark.gpu

UV_TOL = 1e-5


def _items(g):
    nc = int(g["b_nc"])
    return [(g[f"b_P{k}"], g[f"b_T{k}"], g[f"b_U{k}"]) for k in range(nc)]


def _offsets(items):
    return np.cumsum([0] + [len(p) for p, _, _ in items])


def test_batch_sequence_matches_reference(golden, cuda):
    """orient_positive -> arap(6, line search) -> arap(3, free) -> repair_flips,
    the sequence pipeline.py:864-878 runs, against the reference Batch."""
    from ultimate_uv_artist_b200.engine import gpu
    items = _items(golden)
    off = _offsets(items)
    b = gpu.Batch(items)
    b.orient_positive()
    Ua = np.concatenate(b.chart_uvs())
    assert np.abs(Ua - golden["b_Ua"]).max() < 1e-12
    b.arap(6, line_search=True)
    st = b.status()
    assert (st["resid"] <= 1e-6 + 1e-12).all(), st["resid"]
    assert (st["flags"] & 3 == 0).all()
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), golden["b_Ub"], off) < UV_TOL
    b.arap(3, line_search=False)
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), golden["b_Uc"], off) < UV_TOL
    b.U = torch.from_numpy(golden["b_Ud"])
    assert np.array_equal(b.flips_per_chart().cpu().numpy(), golden["b_flips"])
    b.repair_flips(40)
    assert np.abs(np.concatenate(b.chart_uvs()) - golden["b_Ue"]).max() < 1e-9


def test_batch_rhs_and_signed_area(golden, cuda):
    from ultimate_uv_artist_b200.engine import gpu
    items = _items(golden)
    b = gpu.Batch(items)
    b.orient_positive()
    ref = O.BatchRef(items)
    ref.orient_positive()
    sa = b.signed_area().double().cpu().numpy()
    assert np.abs(sa - ref.signed_area(ref.U)).max() < 1e-6 * np.abs(ref.signed_area(ref.U)).max()
    J = b.db.jacobians().cpu().numpy()
    Jr = np.stack(ref.jacobians(ref.U), 1)
    assert np.allclose(J, Jr, rtol=1e-9, atol=1e-9)
    assert abs(float(b.db.wpin[0]) - float(golden["b_wpin"])) < 1e-12


def test_param_lscm_and_refine(golden, cuda):
    """param semantics on one chart: LSCM with the far-pair pins and 10 ARAP
    iterations (tol=0) against engine/param.py run by the reference."""
    from ultimate_uv_artist_b200 import _lib
    from ultimate_uv_artist_b200.device import DeviceBatch
    P, T = golden["p_P"], golden["p_T"]
    n, t = len(P), len(T)
    db = DeviceBatch(P, T, [0, n], [0, t], semantics=_lib.SEM_PARAM)
    assert tuple(db.pins[0, 1:].cpu().tolist()) == tuple(golden["p_pins"].tolist())
    db.lscm()
    U0 = db.uvs()
    ext = np.ptp(golden["p_U0"], 0).max()
    assert np.abs(U0 - golden["p_U0"]).max() / ext < 1e-7
    db.U.copy_(torch.from_numpy(golden["p_U0"]))
    db.arap(iters=10, line_search=True, energy_tol=0.0, tol=1e-11)
    assert np.abs(db.uvs() - golden["p_U1"]).max() / ext < 1e-7
    db.U.copy_(torch.from_numpy(golden["p_U0"]))
    db.arap(iters=10, line_search=True, energy_tol=1e-5, tol=1e-11)
    st = db.island_status()
    assert np.abs(db.uvs() - golden["p_U2"]).max() / ext < 1e-7, st
    db.U.copy_(torch.from_numpy(golden["p_Uf"]))
    db.repair_flips(60, serial=True)
    assert np.abs(db.uvs() - golden["p_Ur"]).max() == 0.0


def test_uneven_batch_lscm_arap_vs_oracle(cuda):
    """A config-2-like batch (log-uniform island sizes up to 20k triangles):
    batched LSCM + 5 ARAP iterations against the FP64 exact-solve oracle."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=77, count=24, tmin=20, tmax=20000)
    b = gpu.Batch([(p, t, None) for p, t in isl])
    b.lscm()
    st = b.status()
    assert (st["flags"] & 3 == 0).all(), st
    U0 = np.concatenate(b.chart_uvs())
    items = [(p.astype(np.float64), t, O.lscm(p.astype(np.float64), t)) for p, t in isl]
    off = _offsets(items)
    assert O.uv_rel_error(U0, np.concatenate([u for _, _, u in items]), off) < UV_TOL
    ref = O.BatchRef(items)
    b.U = torch.from_numpy(ref.U)
    b.arap(5, line_search=True)
    ref.arap(5, line_search=True)
    st = b.status()
    assert (st["resid"] <= 1e-6 + 1e-12).all()
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), ref.U, off) < UV_TOL


def test_lscm_closed_chart_raises(cuda):
    from ultimate_uv_artist_b200.engine import gpu
    # a closed octahedron has no boundary
    P = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    T = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]])
    b = gpu.Batch([(P, T, None)])
    with pytest.raises(ValueError):
        b.lscm()


def test_step_graph_replays_the_direct_calls(cuda):
    """setup + LSCM + 5 ARAP iterations captured once (uva_step_graph_create)
    and replayed twice give the UVs of the same calls made directly: the
    island solver is deterministic (fixed reduction orders, slice-ordered
    coarse restriction), so the comparison is exact."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=77, count=40, tmin=20, tmax=12000)
    b = gpu.Batch([(p, t, None) for p, t in isl])
    db = b.db
    db.setup(); db.lscm(); db.arap(iters=5)
    torch.cuda.synchronize()
    direct = db.U.clone()
    st_direct = db.island_status()
    g = db.step_graph(setup=True, lscm=True, arap_iters=5)
    for _ in range(2):
        db.U.zero_()
        g.launch()
        torch.cuda.synchronize()
        assert torch.equal(db.U, direct)
    st = db.island_status()
    assert np.array_equal(st["cg_iters"], st_direct["cg_iters"])
    assert (st["resid"] <= 1e-6 + 1e-12).all()
    g.close()


def test_large_island_global_memory_class_vs_oracle(cuda):
    """An island above the shared-memory classes (n > 8192 rows: CG vectors
    in L2, 128-row or larger aggregates) next to small ones: LSCM and 4 ARAP
    iterations against the FP64 oracle."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    rng = np.random.default_rng(8)
    isl = [synth.disk_patch(rng, 60000, amp=0.3), synth.disk_patch(rng, 300), synth.disk_patch(rng, 3000)]
    assert len(isl[0][0]) > 8192
    b = gpu.Batch([(p, t, None) for p, t in isl])
    assert int(b.db.plan.class_ofs[1]) == 1          # one island in the global-memory class
    b.lscm()
    items = [(p.astype(np.float64), t, O.lscm(p.astype(np.float64), t)) for p, t in isl]
    off = _offsets(items)
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), np.concatenate([u for _, _, u in items]), off) < UV_TOL
    ref = O.BatchRef(items)
    b.U = torch.from_numpy(ref.U)
    b.arap(4, line_search=True)
    ref.arap(4, line_search=True)
    assert (b.status()["resid"] <= 2e-7 * 1.001).all()
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), ref.U, off) < UV_TOL


def test_wide_class_islands_vs_oracle(cuda):
    """Islands above 16,384 vertices are solved by the whole GPU as one team
    (k_wide, before the persistent launch): two of them, an island of the
    single-CTA global-memory class and small ones. LSCM and 4 ARAP
    iterations against the FP64 oracle; the status names the team; the
    same steps captured in a CUDA graph (the cooperative launch as a graph
    node) give the same UVs bit for bit (every CTA adds the cross-CTA
    partials in the same order)."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    rng = np.random.default_rng(12)
    isl = [synth.disk_patch(rng, 90000, amp=0.3), synth.disk_patch(rng, 300), synth.disk_patch(rng, 50000, amp=0.4),
           synth.disk_patch(rng, 24000), synth.disk_patch(rng, 3000), synth.disk_patch(rng, 40)]
    nv = np.array([len(p) for p, _ in isl])
    wide = nv > 16384
    assert wide.sum() == 2 and ((nv > 8192) & ~wide).sum() == 1
    b = gpu.Batch([(p, t, None) for p, t in isl])
    b.lscm()
    st = b.status()
    assert (st["team"][wide] == 148 * 1024).all() and (st["team"][~wide] <= 1024).all()
    items = [(p.astype(np.float64), t, O.lscm(p.astype(np.float64), t)) for p, t in isl]
    off = _offsets(items)
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), np.concatenate([u for _, _, u in items]), off) < UV_TOL
    ref = O.BatchRef(items)
    b.U = torch.from_numpy(ref.U)
    b.arap(4, line_search=True)
    ref.arap(4, line_search=True)
    st = b.status()
    assert (st["resid"] <= 2e-7 * 1.001).all() and (st["flags"] & 3 == 0).all()
    assert (st["team"][wide] == 148 * 1024).all()
    assert O.uv_rel_error(np.concatenate(b.chart_uvs()), ref.U, off) < UV_TOL
    db = b.db
    db.setup(); db.lscm(); db.arap(iters=4)
    torch.cuda.synchronize()
    direct = db.uvs()
    g = db.step_graph(setup=True, lscm=True, arap_iters=4)
    db.U.zero_()
    g.launch()
    torch.cuda.synchronize()
    g.close()
    st = db.island_status()
    assert (st["resid"] <= 2e-7 * 1.001).all() and (st["team"][wide] == 148 * 1024).all()
    assert np.array_equal(db.uvs(), direct)


def test_batch_edge_cases(cuda):
    """Empty batch; one-triangle and degenerate charts; a chart with
    non-finite UVs keeps them while its neighbours solve normally
    (gpu.py:235-240)."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import gpu
    e = gpu.Batch([])
    e.arap(3)
    assert e.chart_uvs() == []
    rng = np.random.default_rng(9)
    P1 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    T1 = np.array([[0, 1, 2]])
    Pd = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0]], float)   # one zero-area triangle
    Td = np.array([[0, 1, 2], [0, 1, 3]])
    Pg, Tg = synth.disk_patch(rng, 400)
    Pn, Tn = synth.disk_patch(rng, 200)
    Ug = Pg[:, :2].astype(np.float64)
    Un = np.full((len(Pn), 2), np.nan)
    items = [(P1, T1, P1[:, :2].copy()), (Pd, Td, Pd[:, :2].copy()), (Pg, Tg, Ug), (Pn, Tn, Un)]
    b = gpu.Batch(items)
    b.arap(3, line_search=True)
    st = b.status()
    U = b.chart_uvs()
    assert np.isnan(U[3]).all() and st["flags"][3] & 2
    # the degenerate chart's lone vertex has an all-zero row: it keeps its UV
    assert np.isfinite(U[1]).all() and np.array_equal(U[1][2], Pd[2, :2])
    # the oracle's exact LU needs non-singular blocks: compare the other two
    sel = [items[0], items[2]]
    ref = O.BatchRef([(np.asarray(p, np.float64), t, u) for p, t, u in sel])
    ref.arap(3, line_search=True)
    assert O.uv_rel_error(np.concatenate([U[0], U[2]]), ref.U, _offsets(sel)) < UV_TOL


def test_schedule_autotuner(cuda):
    """The autotuner times the candidate team schedules on the batch and
    applies the fastest; the schedule changes which team solves an island,
    not the solution (every island still reaches the tolerance)."""
    from ultimate_uv_artist_b200 import autotune, synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=78, count=60, tmin=20, tmax=6000)
    b = gpu.Batch([(p, t, None) for p, t in isl])
    db = b.db
    db.lscm()
    db.arap(iters=4)
    ref = db.U.clone()
    db.lscm()
    best, res = autotune.tune(db, arap_iters=2)
    assert len(res) == 12 and best == autotune.tune(db)[0]      # second call: cached
    assert (best["mid"], best["small"]) == db.plan.classes
    db.lscm()
    db.arap(iters=4)
    assert (db.island_status()["resid"] <= 2e-7 * 1.001).all()
    # teams of different widths add in different orders: both solutions meet
    # the 2e-7 residual, so they agree to about that level, not bitwise
    ext = float((ref.max(0).values - ref.min(0).values).max())
    assert float((db.U - ref).abs().max()) / ext < 1e-6


def test_start_history_buffer_optional(cuda):
    """Without the batch's history buffer (uva_batch.hist null, as a C caller
    may leave it) the ARAP starts use two updates kept in the class-G CG
    buffers: same tolerance, the same UVs to the solver's accuracy."""
    import ctypes as C
    from ultimate_uv_artist_b200 import _lib, synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=311, count=30, tmin=20, tmax=6000)
    b = gpu.Batch([(p, t, None) for p, t in isl])
    db = b.db
    db.lscm()
    U0 = db.U.clone()
    db.arap(iters=8)
    ref = db.U.clone()
    ext = float((ref.max(0).values - ref.min(0).values).max())
    db.U.copy_(U0)
    desc = _lib.BatchDesc.from_buffer_copy(db.desc)
    desc.hist = None
    prm = db.params("arap", iters=8, line_search=True)
    _lib.check(_lib.lib().uva_arap(C.byref(desc), C.byref(prm), db._stream()), "uva_arap")
    torch.cuda.synchronize()
    assert (db.island_status()["resid"] <= 2e-7 * 1.001).all()
    assert float((db.U - ref).abs().max()) / ext < 1e-5


def test_class_capacity_guard(cuda):
    """An island listed in a team class too small for it (a C caller's
    inconsistent class_ofs) is refused with UVA_ST_BADCLASS and left
    untouched; the islands that fit are solved."""
    import ctypes as C
    from ultimate_uv_artist_b200 import _lib, synth
    from ultimate_uv_artist_b200.engine import gpu
    isl = synth.uneven_islands(seed=312, count=12, tmin=20, tmax=2000)
    b = gpu.Batch([(p, t, None) for p, t in isl])
    db = b.db
    db.lscm()
    U0 = db.U.clone()
    desc = _lib.BatchDesc.from_buffer_copy(db.desc)
    for c in range(3):   # every island to the one-warp class (256 rows at most)
        desc.class_ofs[c] = 0
    desc.class_ofs[3] = 0
    desc.class_ofs[4] = db.nc
    prm = db.params("arap", iters=3, line_search=True)
    _lib.check(_lib.lib().uva_arap(C.byref(desc), C.byref(prm), db._stream()), "uva_arap")
    torch.cuda.synchronize()
    st = db.island_status()
    n = np.diff(db.plan.vofs)
    big = n > 256
    assert big.any() and (~big).any()
    assert ((st["flags"][big] & _lib.ST_BADCLASS) != 0).all()
    assert ((st["flags"][~big] & _lib.ST_BADCLASS) == 0).all()
    assert (st["resid"][~big] <= 2e-7 * 1.001).all()
    vofs = db.plan.vofs.astype(np.int64)
    for i in np.where(big)[0]:
        a, e = vofs[i], vofs[i + 1]
        assert torch.equal(db.U[a:e], U0[a:e])
