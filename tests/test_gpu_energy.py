"""Hand-written backward kernels of the ARAP and symmetric-Dirichlet energies
(engine/param.py:294-319), checked against FP64 central finite differences
(h = 1e-6), against the ARAP identity grad_U E = 2 (L U - b(R(U))) built by
the oracle from the reference's formulas, and driving 50 steps of p95-stretch
refinement."""
import numpy as np
import pytest
import torch

from oracle import arap as O

pytestmark = pytest.mark.gpu


def _batch(islands, U=None):
    from ultimate_uv_artist_b200 import _lib
    from ultimate_uv_artist_b200.device import DeviceBatch, concat_charts
    P, T, Uc, vofs, tofs = concat_charts([(p, t) for p, t in islands], with_uv=False)
    if U is None:
        U = P[:, :2].copy()     # graph patches: the xy projection is flip-free
    return DeviceBatch(P, T, vofs, tofs, U=U, semantics=_lib.SEM_PARAM), P, T, U, vofs, tofs


def _oracle_energy(P, T, U, vofs, tofs, kind):
    out = []
    for i in range(len(vofs) - 1):
        Ti = T[tofs[i]:tofs[i + 1]]
        Pi, Ui = P[vofs[i]:vofs[i + 1]], U[vofs[i]:vofs[i + 1]]
        X, area = O.local_frames(Pi, Ti)
        out.append(O.energy(Ui, Ti, X, area, kind))
    return np.array(out)


def test_gradcheck_central_differences(cuda):
    """torch.autograd.gradcheck: FP64 central differences, eps = 1e-6."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.energy import DistortionEnergy
    rng = np.random.default_rng(3)
    isl = [synth.disk_patch(rng, 24, amp=0.3), synth.disk_patch(rng, 40, amp=0.3)]
    db, P, T, U, vofs, tofs = _batch(isl)
    Ut = torch.from_numpy(U + rng.normal(0, 0.01, U.shape)).to(cuda).requires_grad_(True)
    Pt = torch.from_numpy(P.copy()).to(cuda).requires_grad_(True)
    # the backward adds the corner terms with FP64 atomics, so two backward
    # passes may differ in the last bits (summation order): nondet_tol allows
    # that round-off, nothing more
    for kind in (0, 1):
        assert torch.autograd.gradcheck(lambda u, p: DistortionEnergy.apply(u, p, db, kind), (Ut, Pt), eps=1e-6,
                                        atol=1e-6, rtol=1e-5, nondet_tol=1e-12)


def test_energy_values_and_fd_on_near_degenerate_islands(cuda):
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.energy import distortion_energy
    isl = synth.energy_islands(seed=4000, count=4, tmin=500, tmax=3000)
    db, P, T, U, vofs, tofs = _batch(isl)
    for kind in (0, 1):
        e = distortion_energy(db, kind=kind).cpu().numpy()
        ref = _oracle_energy(P, T, U, vofs, tofs, kind)
        assert np.allclose(e, ref, rtol=1e-10), (kind, e, ref)
    # gradients against FP64 central differences at sampled coordinates. Near
    # the aspect-1e3 triangles the h = 1e-6 difference still carries an h^2
    # truncation term (it shrinks 100x per decade of h), so the check uses
    # Richardson extrapolation of the h = 1e-6 and h = 5e-7 differences.
    Ut = torch.from_numpy(U).to(cuda).requires_grad_(True)
    Pt = torch.from_numpy(P).to(cuda).requires_grad_(True)
    rng = np.random.default_rng(0)

    def fd(arr, v, c, dim, kind, h):
        Xp = arr.copy(); Xp[v, c] += h
        Xm = arr.copy(); Xm[v, c] -= h
        if dim == 2:
            return (_oracle_energy(P, T, Xp, vofs, tofs, kind).sum() - _oracle_energy(P, T, Xm, vofs, tofs, kind).sum()) / (2 * h)
        return (_oracle_energy(Xp, T, U, vofs, tofs, kind).sum() - _oracle_energy(Xm, T, U, vofs, tofs, kind).sum()) / (2 * h)

    for kind in (0, 1):
        E = distortion_energy(db, Ut, Pt, kind=kind).sum()
        gU, gP = torch.autograd.grad(E, (Ut, Pt))
        gU, gP = gU.cpu().numpy(), gP.cpu().numpy()
        worst = worst_plain = 0.0
        for arr, g, dim in ((U, gU, 2), (P, gP, 3)):
            for idx in rng.choice(arr.size, 30, replace=False):
                v, c = divmod(int(idx), dim)
                f1 = fd(arr, v, c, dim, kind, 1e-6)
                f2 = fd(arr, v, c, dim, kind, 5e-7)
                rich = (4.0 * f2 - f1) / 3.0
                scale = max(abs(rich), 1e-3 * np.abs(g).max())
                worst = max(worst, abs(g[v, c] - rich) / scale)
                worst_plain = max(worst_plain, abs(g[v, c] - f1) / scale)
        assert worst < 1e-5, (kind, worst)
        assert worst_plain < 1e-2, (kind, worst_plain)


def test_arap_gradient_identity(cuda):
    """grad_U E_ARAP = 2 (L U - b(R(U))) with L the cotangent Laplacian and b
    the ARAP right-hand side of engine/param.py (oracle restatement)."""
    import scipy.sparse as sp
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.energy import distortion_energy
    isl = synth.energy_islands(seed=4001, count=2, tmin=300, tmax=800)
    rng = np.random.default_rng(5)
    db, P, T, U, vofs, tofs = _batch(isl)
    U = U + rng.normal(0, 0.02, U.shape)
    Ut = torch.from_numpy(U).to(cuda).requires_grad_(True)
    E = distortion_energy(db, Ut, kind=0).sum()
    (gU,) = torch.autograd.grad(E, (Ut,))
    gU = gU.cpu().numpy()
    for i in range(len(vofs) - 1):
        Ti = T[tofs[i]:tofs[i + 1]]
        Pi, Ui = P[vofs[i]:vofs[i + 1]], U[vofs[i]:vofs[i + 1]]
        X, _ = O.local_frames(Pi, Ti)
        cots = O.cot_weights(X)
        I, J, W = O.lap_triplets(Ti, cots)
        L = sp.csr_matrix((W, (I, J)), shape=(len(Pi), len(Pi)))
        b = O.arap_rhs(len(Pi), Ti, X, cots, O.arap_rotations(Ui, Ti, X))
        ref = 2.0 * (L @ Ui - b)
        g = gU[vofs[i]:vofs[i + 1]]
        assert np.abs(g - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1.0), np.abs(g - ref).max()


def test_sd_refinement_lowers_p95_stretch(cuda):
    """50 steps of p95-stretch refinement: per-island symmetric Dirichlet
    energies never increase, no fold appears, p95 anisotropy drops."""
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.energy import distortion_energy, sd_refine
    from ultimate_uv_artist_b200.engine import param as Pm
    isl = synth.energy_islands(seed=4002, count=6, tmin=500, tmax=5000)
    db, P, T, U, vofs, tofs = _batch(isl)
    e0 = distortion_energy(db, kind=1).cpu().numpy()
    q0 = [q["aniso_p95"] for q in Pm.chart_quality_batch(db)]
    e1 = sd_refine(db, steps=50).cpu().numpy()
    q1 = [q["aniso_p95"] for q in Pm.chart_quality_batch(db)]
    assert np.isfinite(e1).all() and (e1 <= e0 + 1e-12 * np.abs(e0)).all()
    assert (e1 < e0).any()
    sa = db.signed_area().cpu().numpy()
    assert (sa > 0).all()
    assert np.mean(q1) < np.mean(q0), (q0, q1)


def test_config4_energies_full_size(cuda):
    """Config 4 at its stated size: 512 islands of 500 to 50,000 triangles
    (5.8M in total) with 5 % near-degenerate triangles (aspect up to 1e3).
    * ARAP and symmetric-Dirichlet energies of every island against the FP64
      oracle (1e-10 relative) on 16 size-stratified islands;
    * gradients with respect to U and P against FP64 central differences
      (h = 1e-6, Richardson-extrapolated with h = 5e-7) at 48 coordinates
      sampled across all islands, each difference taken on its own island's
      energy;
    * the ARAP gradient identity 2 (L U - b(R(U))) on 4 stratified islands;
    * 50 steps of p95-stretch refinement: no island's energy rises, no fold
      appears, and the p95 anisotropy (param.chart_quality) is compared with
      the reference's SLIM refinement (param.refine(method="slim"), 15
      iterations as in the "artist" profile) run from the same start on the
      same islands; uva_slim itself matches the oracle's SLIM on 2 islands."""
    import scipy.sparse as sp
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.energy import distortion_energy, sd_refine
    from ultimate_uv_artist_b200.engine import param as Pm
    isl = synth.energy_islands(seed=4000, count=512, tmin=500, tmax=50000)
    db, P, T, U, vofs, tofs = _batch(isl)
    assert db.t > 5_000_000
    nt = np.diff(tofs)
    order = np.argsort(nt)
    pick = order[np.linspace(0, len(order) - 1, 16).astype(int)]
    for kind in (0, 1):
        e = distortion_energy(db, kind=kind).cpu().numpy()
        for i in pick:
            Ti, Pi, Ui = T[tofs[i]:tofs[i + 1]], P[vofs[i]:vofs[i + 1]], U[vofs[i]:vofs[i + 1]]
            X, area = O.local_frames(Pi, Ti)
            assert abs(e[i] - O.energy(Ui, Ti, X, area, kind)) <= 1e-10 * abs(e[i]), (kind, i)
    # gradients against central differences, coordinates sampled over all islands
    Ut = torch.from_numpy(U).to(cuda).requires_grad_(True)
    Pt = torch.from_numpy(P).to(cuda).requires_grad_(True)
    isl_of_v = np.repeat(np.arange(len(vofs) - 1), np.diff(vofs))
    rng = np.random.default_rng(4)

    def island_energy(i, Pi, Ui, kind):
        Ti = T[tofs[i]:tofs[i + 1]]
        X, area = O.local_frames(Pi, Ti)
        return O.energy(Ui, Ti, X, area, kind)

    def fd(i, v, c, wrt, kind, h):
        Pi, Ui = P[vofs[i]:vofs[i + 1]].copy(), U[vofs[i]:vofs[i + 1]].copy()
        A = Ui if wrt == "U" else Pi
        A[v, c] += h
        fp = island_energy(i, Pi, Ui, kind)
        A[v, c] -= 2 * h
        fm = island_energy(i, Pi, Ui, kind)
        return (fp - fm) / (2 * h)

    for kind in (0, 1):
        E = distortion_energy(db, Ut, Pt, kind=kind).sum()
        gU, gP = torch.autograd.grad(E, (Ut, Pt))
        gU, gP = gU.cpu().numpy(), gP.cpu().numpy()
        worst = 0.0
        for wrt, g, dim in (("U", gU, 2), ("P", gP, 3)):
            for vg in rng.choice(db.n, 24, replace=False):
                i = int(isl_of_v[vg])
                v = int(vg - vofs[i])
                c = int(rng.integers(dim))
                f1, f2 = fd(i, v, c, wrt, kind, 1e-6), fd(i, v, c, wrt, kind, 5e-7)
                rich = (4.0 * f2 - f1) / 3.0
                gi = g[vofs[i]:vofs[i + 1]]
                scale = max(abs(rich), 1e-3 * np.abs(gi).max())
                worst = max(worst, abs(g[vg, c] - rich) / scale)
        assert worst < 1e-5, (kind, worst)
    # the ARAP identity on stratified islands
    gU = torch.autograd.grad(distortion_energy(db, Ut, kind=0).sum(), (Ut,))[0].cpu().numpy()
    for i in pick[::4]:
        Ti, Pi, Ui = T[tofs[i]:tofs[i + 1]], P[vofs[i]:vofs[i + 1]], U[vofs[i]:vofs[i + 1]]
        X, _ = O.local_frames(Pi, Ti)
        cots = O.cot_weights(X)
        I, J, W = O.lap_triplets(Ti, cots)
        L = sp.csr_matrix((W, (I, J)), shape=(len(Pi), len(Pi)))
        ref = 2.0 * (L @ Ui - O.arap_rhs(len(Pi), Ti, X, cots, O.arap_rotations(Ui, Ti, X)))
        g = gU[vofs[i]:vofs[i + 1]]
        # the identity needs the exact cotangents: rows touching a triangle
        # whose cotangent the reference clips at +-1e4 are left out
        clipped = np.zeros(len(Pi), bool)
        clipped[Ti[(np.abs(cots) >= 1e4).any(1)].ravel()] = True
        assert np.abs(g - ref)[~clipped].max() <= 1e-9 * max(np.abs(ref).max(), 1.0)
    # 50 refinement steps against SLIM from the same start
    q0 = np.array([q["aniso_p95"] for q in Pm.chart_quality_batch(db)])
    e0 = distortion_energy(db, kind=1).cpu().numpy()
    e1 = sd_refine(db, steps=50).cpu().numpy()
    assert np.isfinite(e1).all() and (e1 <= e0 + 1e-12 * np.abs(e0)).all()
    assert (db.signed_area().cpu().numpy() > 0).all()
    q1 = np.array([q["aniso_p95"] for q in Pm.chart_quality_batch(db)])
    assert np.median(q1) < np.median(q0)
    # SLIM (one CTA per island, exact-solve tolerance) on the 12 smaller of
    # the stratified islands (up to about 20k triangles), from the same start
    sub_idx = pick[:12]
    ds, Ps, Ts, Us0, vs, ts = _batch([isl[i] for i in sub_idx])
    ds.slim(iters=15, cg_tol=1e-12)
    qs = np.array([q["aniso_p95"] for q in Pm.chart_quality_batch(ds)])
    print(f"config4 p95 anisotropy, 12 stratified islands (median): start {np.median(q0[sub_idx]):.4f}, "
          f"sd_refine(50) {np.median(q1[sub_idx]):.4f}, SLIM(15) {np.median(qs):.4f}; "
          f"all 512: start {np.median(q0):.4f}, sd_refine(50) {np.median(q1):.4f}")
    # uva_slim restates the reference's SLIM: its p95 anisotropy against the
    # oracle's on two islands. With aspect-1e3 triangles the SLIM normal
    # equations are ill-conditioned (the translation is fixed only by a
    # 1e-12 sum(area) regulariser), so the UVs of an iterative and an exact
    # solve drift apart (4e-4 of the extent here); the UV bar of SLIM is
    # checked on well-shaped charts against the reference's own output
    # (test_gpu_metrics_param.py::test_slim_rotations_and_refine).
    Ug = ds.uvs()
    for k in (2, 8):
        Ti, Pi, Ui = Ts[ts[k]:ts[k + 1]], Ps[vs[k]:vs[k + 1]], Us0[vs[k]:vs[k + 1]]
        R = O.refine_slim(Pi, Ti, Ui, iters=15)
        qr = O.chart_quality(Pi, Ti, R)["aniso_p95"]
        qg = O.chart_quality(Pi, Ti, Ug[vs[k]:vs[k + 1]])["aniso_p95"]
        assert abs(qg - qr) <= 1e-3 * qr, (k, qg, qr)
