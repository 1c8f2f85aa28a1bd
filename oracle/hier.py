"""Oracle for hier.Solver (test infrastructure only): FP64 restatements of
engine/hier.py:357-593 with exact global solves.

* ``relax``: per-chart batch (oracle.arap.BatchRef, exact sparse LU), the
  reference's sequence: orientation, flip repair, ARAP iterations with the
  step rule of engine/hier.py:541-555 (flip-safe step, full step for charts
  folded at the start of the iteration), repair after iteration iters // 2
  and at the end, then the per-chart quality of :493-508.
* ``lscm``: the soft-pinned LSCM system of engine/hier.py:511-583, solved
  exactly (scipy spsolve). Pins: per chart, the boundary vertices of
  smallest and largest initial u compared in float32 (the reference's key
  dtype), the smallest vertex id on ties.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.arap import BatchRef


def _vchart(CV, chart, nv):
    vchart = -np.ones(nv, np.int64)
    for i in range(len(CV)):
        for k in range(3):
            vchart[CV[i, k]] = chart[i]
    return vchart


def layout(V, F, faces, CV, nv, chart, nchart, U0):
    """Charts as (P, T_local, U) islands, vertices by chart then id; returns
    the charts and the batch order of the UV vertices."""
    vchart = _vchart(CV, chart, nv)
    charts, order = [], []
    for c in range(nchart):
        vs = np.nonzero(vchart == c)[0]
        loc = {int(v): k for k, v in enumerate(vs)}
        fs = np.nonzero(chart == c)[0]
        T = np.array([[loc[int(v)] for v in CV[i]] for i in fs], np.int64).reshape(-1, 3)
        P = np.empty((len(vs), 3))
        for i in fs:
            for k in range(3):
                P[loc[int(CV[i, k])]] = V[F[faces[i], k]]
        charts.append((P, T, U0[vs].copy()))
        order.append(vs)
    return charts, np.concatenate(order) if order else np.zeros(0, np.int64)


def relax(V, F, faces, CV, nv, chart, nchart, U0, iters=6, repair_rounds=24):
    """engine/hier.py:389-509 with exact solves -> (U, flips, scale, q)."""
    V = np.asarray(V, np.float64); F = np.asarray(F, np.int64)
    CV = np.asarray(CV, np.int64); chart = np.asarray(chart, np.int64)
    U0 = np.asarray(U0, np.float64)
    charts, order = layout(V, F, faces, CV, nv, chart, nchart, U0)
    ref = BatchRef(charts)
    ref.orient_positive()
    ref.repair_flips(repair_rounds)
    U = ref.U
    for it in range(iters):
        b = ref.rhs(U)
        Un = ref._solve(b)
        badv = ~np.isfinite(Un).all(1)
        if badv.any():
            badc = np.zeros(ref.nc, bool)
            badc[ref.cv[badv]] = True
            Un = np.where(badc[ref.cv][:, None], U, Un)
        flipped = (ref.signed_area(U) < 0) & ref.ok
        fl_c = np.bincount(ref.ct, weights=flipped.astype(float), minlength=ref.nc)
        D = Un - U
        step = np.minimum(0.9 * ref.max_step(U, D), 1.0)
        step = np.where(fl_c > 0, 1.0, step)
        U = U + D * step[ref.cv][:, None]
        if it == iters // 2:
            ref.U = U
            U = ref.repair_flips(repair_rounds)
    ref.U = U
    U = ref.repair_flips(repair_rounds)
    j00, j01, j10, j11 = ref.jacobians(U)
    E = (j00 + j11) / 2; Fq = (j00 - j11) / 2; G = (j10 + j01) / 2; H = (j10 - j01) / 2
    Q = np.sqrt(E * E + H * H); R = np.sqrt(Fq * Fq + G * G)
    s1 = Q + R; s2 = np.abs(Q - R)
    ok = ref.ok
    ar3 = ref.area * ok
    sgn = ref.signed_area(U)
    uva = np.bincount(ref.ct, np.abs(sgn) * ok, ref.nc)
    a3 = np.bincount(ref.ct, ar3, ref.nc)
    scale = uva / np.maximum(a3, 1e-30)
    with np.errstate(divide="ignore", invalid="ignore"):
        aniso = s1 / np.maximum(s2, 1e-12)
        arat = (s1 * s2) / np.maximum(scale[ref.ct], 1e-30)
    flips = np.bincount(ref.ct, ((sgn < 0) & ok).astype(float), ref.nc)
    out = U0.copy()
    out[order] = U
    return out, flips, scale, (aniso, arat, ar3, ref.ct, ref.nc, a3)


def bad_fraction(q, max_aniso, max_area):
    """engine/hier.py:585-591."""
    aniso, arat, ar3, ct, nchart, a3 = q
    badA = np.bincount(ct, ar3 * (aniso > max_aniso), nchart)
    badR = np.bincount(ct, ar3 * ((arat > max_area) | (arat < 1.0 / max_area)), nchart)
    return badA / np.maximum(a3, 1e-30), badR / np.maximum(a3, 1e-30)


def face_cots(V, Ff):
    """engine/hier.py:362-382 in FP64."""
    p0, p1, p2 = V[Ff[:, 0]], V[Ff[:, 1]], V[Ff[:, 2]]
    e1 = p1 - p0; e2 = p2 - p0
    l1 = np.linalg.norm(e1, axis=1)
    nrm = np.cross(e1, e2)
    dbl = np.linalg.norm(nrm, axis=1)
    ok = (dbl > 1e-14 * np.maximum(l1 * l1, 1e-300)) & np.isfinite(dbl) & (l1 > 0)
    ex = e1 / np.maximum(l1, 1e-30)[:, None]
    ey = np.cross(nrm / np.maximum(dbl, 1e-30)[:, None], ex)
    X = np.zeros((len(Ff), 3, 2))
    X[:, 1, 0] = l1; X[:, 2, 0] = (e2 * ex).sum(1); X[:, 2, 1] = (e2 * ey).sum(1)
    X[~ok] = 0
    w = np.zeros((len(Ff), 3))
    for k in range(3):
        i, j, o = (k + 1) % 3, (k + 2) % 3, k
        a = X[:, i] - X[:, o]; b = X[:, j] - X[:, o]
        cr = np.maximum(np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]), 1e-30)
        w[:, k] = 0.5 * np.clip((a * b).sum(1) / cr, -1e4, 1e4)
    w[~ok] = 0
    return w


def lscm_pins(CV, chart, nv, U0, ba):
    """Per chart: the boundary vertices of smallest and largest initial u
    (float32 keys, smallest id on ties)."""
    vchart = _vchart(CV, chart, nv)
    bv = np.unique(np.asarray(ba, np.int64))
    key = U0[bv, 0].astype(np.float32)
    p0, p1 = {}, {}
    for v, k in zip(bv.tolist(), key.tolist()):
        c = int(vchart[v])
        if c not in p0 or k < p0[c][0]:
            p0[c] = (k, v)
        if c not in p1 or k > p1[c][0]:
            p1[c] = (k, v)
    return np.array([p0[c][1] for c in sorted(p0)] + [p1[c][1] for c in sorted(p1)], np.int64)


def lscm(V, F, faces, CV, nv, chart, nchart, U0, ba, bb):
    """engine/hier.py:511-583, exact solve of the soft-pinned system."""
    V = np.asarray(V, np.float64); F = np.asarray(F, np.int64)
    CV = np.asarray(CV, np.int64); U0 = np.asarray(U0, np.float64)
    ba = np.asarray(ba, np.int64); bb = np.asarray(bb, np.int64)
    w = face_cots(V, F[np.asarray(faces, np.int64)])
    I = np.concatenate([CV[:, 1], CV[:, 2], CV[:, 0]])
    J = np.concatenate([CV[:, 2], CV[:, 0], CV[:, 1]])
    Wl = np.concatenate([w[:, 0], w[:, 1], w[:, 2]])
    hb = np.full(len(ba), 0.5)
    pins = lscm_pins(CV, chart, nv, U0, ba)
    wpin = max(np.abs(Wl).max(), 1e-12) * 10
    rows = np.concatenate([I, J, I, J, I + nv, J + nv, I + nv, J + nv, ba, bb, ba + nv, bb + nv, pins, pins + nv])
    cols = np.concatenate([J, I, I, J, J + nv, I + nv, I + nv, J + nv, bb + nv, ba + nv, bb, ba, pins, pins + nv])
    vals = np.concatenate([-Wl, -Wl, Wl, Wl, -Wl, -Wl, Wl, Wl, -hb, hb, hb, -hb, np.full(2 * len(pins), wpin)])
    H = sp.csc_matrix((vals, (rows, cols)), shape=(2 * nv, 2 * nv))
    b = np.zeros(2 * nv)
    np.add.at(b, pins, wpin * U0[pins, 0])
    np.add.at(b, pins + nv, wpin * U0[pins, 1])
    used = np.zeros(2 * nv, bool)
    used[np.unique(np.r_[CV.reshape(-1), CV.reshape(-1) + nv])] = True
    x = np.concatenate([U0[:, 0], U0[:, 1]])
    idx = np.nonzero(used)[0]
    x[idx] = spla.spsolve(H[idx][:, idx].tocsc(), b[idx])
    return np.stack([x[:nv], x[nv:]], 1)
