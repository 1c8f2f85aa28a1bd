"""Generate the golden fixtures of the parameterization / validation path by
running the REFERENCE implementation (Ultimate UV Artist, engine/*.py) on small
seeded inputs.

Run in a checkout that has the reference next to it:

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden.py /path/to/ultimate_uv_artist

The reference is only read here, never at test time: the fixtures (*.npz) are
committed and the tests compare the oracle and the CUDA path against them.
The batched solver fixture runs the reference ``gpu.Batch`` on CPU torch in
float64 with its CG tolerance tightened to 1e-12 (5,000 iterations), so its
global steps are exact solves up to round-off.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ultimate_uv_artist_b200 import synth  # noqa: E402


def small_islands(seed, counts):
    rng = np.random.default_rng(seed)
    return [synth.disk_patch(rng, t) for t in counts]


def main(ref_root):
    sys.path.insert(0, ref_root)
    import torch
    from engine import gpu, metrics, param, validate

    out = {}
    # ------------------------------------------------------------ param path
    P, T = synth.hemisphere_patch(seed=11, n=14, jitter=0.01)
    P = P.astype(np.float64)
    X, area = param.local_frames(P, T)
    cots = param.cot_weights(X)
    U0 = param.lscm(P, T, X, cots)
    bi, _ = param.boundary_edges_oriented(T)
    pins = param._far_pair(P, np.unique(bi))
    U1, _ = param.refine(P, T, U0, iters=10, method="arap", X=X, area=area, cots=cots, line_search=True, tol=0.0)
    U2, _ = param.refine(P, T, U0, iters=10, method="arap", line_search=True, tol=1e-5)
    q = param.chart_quality(P, T, U1, X, area)
    R, _ = param._arap_rotations(U0, T, X, cots, 0, np.empty(0))
    b = param._arap_rhs(len(P), T, X, cots, R)
    # a folded start for repair
    Uf = U1.copy()
    interior = np.setdiff1d(np.arange(len(P)), np.unique(np.r_[param.boundary_edges_oriented(T)]))
    rng = np.random.default_rng(5)
    mv = rng.choice(interior, 4, replace=False)
    for v in mv:
        # push the vertex past a neighbour: folds its fan
        nb = T[(T == v).any(1)].ravel()
        w = nb[nb != v][0]
        Uf[v] = Uf[v] + 2.5 * (Uf[w] - Uf[v])
    Ur = param.repair_flips(Uf, T, rounds=60)
    D = U1 - U0
    out.update(p_P=P, p_T=T, p_X=X, p_area=area, p_cots=cots, p_U0=U0, p_pins=np.array(pins),
               p_U1=U1, p_U2=U2, p_R=R, p_b=b, p_Uf=Uf, p_Ur=Ur,
               p_maxstep=np.array(param._max_step(U0, D, T)),
               p_E0=np.array(param._energy(U1, T, X, area, 0)), p_E1=np.array(param._energy(U1, T, X, area, 1)),
               p_q_aniso_p95=np.array(q["aniso_p95"]), p_q_area_p95=np.array(q["area_p95"]),
               p_q_flips=np.array(q["flips"]), p_q_stretch=np.array(q["stretch"]),
               p_q_aniso=q["per_tri_aniso"], p_q_area=q["per_tri_area"])

    # ------------------------------------------------------------ batch path
    orig = gpu.Batch._cg

    def tight(self, b, x, iters=40, tol=1e-6):
        return orig(self, b, x, iters=5000, tol=1e-12)

    gpu.Batch._cg = tight
    isl = small_islands(21, [20, 60, 150, 400, 900])
    isl.append(synth.hemisphere_patch(seed=12, n=10, jitter=0.01))
    items = []
    for Pi, Ti in isl:
        Pi = Pi.astype(np.float64)
        items.append((Pi, Ti, param.lscm(Pi, Ti)))
    bt = gpu.Batch(items, dev=torch.device("cpu"), dtype=torch.float64)
    bt.orient_positive()
    Ua = bt.U.numpy().copy()
    rhs0 = bt._rhs(bt.U).numpy()
    bt.arap(6, line_search=True)
    Ub = bt.U.numpy().copy()
    bt.arap(3, line_search=False)
    Uc = bt.U.numpy().copy()
    # a fold for Batch.repair_flips
    Ud = Uc.copy()
    rng = np.random.default_rng(7)
    off = bt.offsets
    T3 = items[3][1]
    inner3 = np.setdiff1d(np.arange(off[4] - off[3]), np.unique(np.r_[param.boundary_edges_oriented(T3)]))
    for v in rng.choice(inner3, 3, replace=False):
        nb = T3[(T3 == v).any(1)].ravel()
        w = nb[nb != v][0]
        Ud[off[3] + v] = Ud[off[3] + v] + 2.5 * (Ud[off[3] + w] - Ud[off[3] + v])
    bt.U = torch.from_numpy(Ud.copy())
    fl = bt.flips_per_chart().numpy()
    bt.repair_flips(40)
    Ue = bt.U.numpy().copy()
    gpu.Batch._cg = orig
    for k, (Pi, Ti, Ui) in enumerate(items):
        out[f"b_P{k}"] = Pi; out[f"b_T{k}"] = Ti; out[f"b_U{k}"] = Ui
    out.update(b_nc=np.array(len(items)), b_Ua=Ua, b_rhs0=rhs0, b_Ub=Ub, b_Uc=Uc, b_Ud=Ud, b_flips=fl, b_Ue=Ue,
               b_wpin=np.array(float(bt.wpin)))

    # ------------------------------------------------------------ validation path
    V, F, UV, info = synth.validation_atlas(seed=31, islands=60, tris_per_island=50, atlas=512, padding=4,
                                            overlap_rate=2e-3, fold_rate=2e-3, mirrored=2, outside=5)
    rep, problems = validate.validate_uvs(V, F, UV, atlas=512, padding=4)
    U64 = UV.astype(np.float32).astype(np.float64)
    isl_lab, n_isl = metrics.uv_islands(F, len(V), U64, V)
    p0, p1, p2 = V.astype(np.float64)[F[:, 0]], V.astype(np.float64)[F[:, 1]], V.astype(np.float64)[F[:, 2]]
    a3 = 0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1)
    u = U64[F]
    sa = 0.5 * ((u[:, 1, 0] - u[:, 0, 0]) * (u[:, 2, 1] - u[:, 0, 1]) - (u[:, 2, 0] - u[:, 0, 0]) * (u[:, 1, 1] - u[:, 0, 1]))
    edge = np.maximum(np.maximum(np.linalg.norm(u[:, 1] - u[:, 0], axis=1), np.linalg.norm(u[:, 2] - u[:, 1], axis=1)),
                      np.linalg.norm(u[:, 0] - u[:, 2], axis=1))
    sliver = np.abs(sa) < 2.0 ** -24 * np.maximum(edge, 2.0 ** -24)
    has3d = a3 > 1e-14 * max(float(a3.max()), 1e-30)
    skip = ~has3d | sliver | ~np.isfinite(sa)
    G = int(np.clip(np.sqrt(len(F)) / 2, 64, 4096))
    ov = validate._overlaps(np.ascontiguousarray(U64), np.ascontiguousarray(F), skip, G, 1e-6, 0)
    ovs = validate._overlaps_strict(np.ascontiguousarray(U64), np.ascontiguousarray(F), skip, G)
    g, img = metrics.min_gutter(U64, F, isl_lab, 512)
    dist = metrics.distortion_report(V, F, UV.astype(np.float64), isl_lab)
    s1, s2, sgn, A3, good = metrics.triangle_jacobians(V.astype(np.float64)[F], UV.astype(np.float64)[F])
    counts = np.zeros((256, 256), np.uint8)
    metrics._raster_counts(np.ascontiguousarray(U64), np.ascontiguousarray(F), 256, counts)
    # per-chart overlap on one island with an injected fold
    fchart = F[info["tofs"][0]:info["tofs"][1]] - info["vofs"][0]
    uchart = U64[info["vofs"][0]:info["vofs"][1]].copy()
    uchart[5] += np.array([0.004, 0.003])
    cov = validate.chart_overlaps(uchart, fchart)
    # a clean atlas (one mirrored island, no overlaps): non-zero gutter
    V2, F2, UV2, _ = synth.validation_atlas(seed=33, islands=40, tris_per_island=50, atlas=512, padding=4,
                                            overlap_rate=0.0, fold_rate=0.0, mirrored=1, outside=0)
    rep2, prob2 = validate.validate_uvs(V2, F2, UV2, atlas=512, padding=4)
    U2_64 = UV2.astype(np.float32).astype(np.float64)
    isl2, _ = metrics.uv_islands(F2, len(V2), U2_64, V2)
    g2, img2 = metrics.min_gutter(U2_64, F2, isl2, 512)
    keys2 = sorted(k for k in rep2 if isinstance(rep2[k], (int, float, bool, np.integer, np.floating)))
    out.update(w_V=V2, w_F=F2, w_UV=UV2, w_problems=prob2, w_isl=isl2, w_gutter=np.array(g2),
               w_img=img2.astype(np.int32), w_rep_keys=np.array(keys2),
               w_rep_vals=np.array([float(rep2[k]) for k in keys2]))
    keys = sorted(k for k in rep if isinstance(rep[k], (int, float, bool, np.integer, np.floating)))
    out.update(v_V=V, v_F=F, v_UV=UV, v_problems=problems, v_ov=ov, v_ovs=ovs, v_isl=isl_lab,
               v_nisl=np.array(n_isl), v_gutter=np.array(g), v_img=img.astype(np.int32),
               v_rep_keys=np.array(keys), v_rep_vals=np.array([float(rep[k]) for k in keys]),
               v_dist_keys=np.array(sorted(dist)), v_dist_vals=np.array([float(dist[k]) for k in sorted(dist)]),
               v_s1=s1, v_s2=s2, v_sa=sgn, v_A3=A3, v_good=good, v_counts=counts,
               v_cF=fchart, v_cU=uchart, v_cov=cov)
    # ------------------------------------------------------------ SLIM (artist profile)
    rng = np.random.default_rng(21)
    Ps, Ts = synth.disk_patch(rng, 600, amp=0.3)
    Ps = Ps.astype(np.float64)
    Us0 = param.lscm(Ps, Ts)
    Xs, areas = param.local_frames(Ps, Ts)
    cotss = param.cot_weights(Xs)
    assert np.isfinite(param._energy(Us0, Ts, Xs, areas, 1)), "SLIM fixture needs a flip-free start"
    Rs1, Ws1 = param._arap_rotations(Us0, Ts, Xs, cotss, 1, np.empty(0))
    Us5, _ = param.refine(Ps, Ts, Us0, iters=5, method="slim", tol=0.0)
    Us20, _ = param.refine(Ps, Ts, Us0, iters=20, method="slim")
    out.update(s_P=Ps, s_T=Ts, s_U0=Us0, s_R1=Rs1, s_W1=Ws1, s_U5=Us5, s_U20=Us20,
               s_E0=np.array(param._energy(Us0, Ts, Xs, areas, 1)),
               s_E5=np.array(param._energy(Us5, Ts, Xs, areas, 1)),
               s_E20=np.array(param._energy(Us20, Ts, Xs, areas, 1)))
    path = os.path.join(HERE, "golden_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
