"""Generate the golden fixtures of the boundary self-intersection checks by
running the REFERENCE implementation (Ultimate UV Artist:
engine/charts.py boundary_intersections, engine/hier.py charts_collide,
chart_checks and boundary_directed) on small seeded inputs.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden_segments.py /path/to/ultimate_uv_artist

The reference is only read here, never at test time: the inputs and the
reference's outputs are stored in golden_segments.npz next to this script.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ultimate_uv_artist_b200 import synth  # noqa: E402

MAX_REPORTS = (1, 3, 1000)


# ------------------------------------------------------------------ inputs
def star_chart(rng, k, turns, noise):
    """Fan triangulation of a closed polygon that winds `turns` times around
    the centre: its boundary crosses itself many times."""
    ang = np.linspace(0.0, 2 * np.pi * turns, k, endpoint=False)
    r = 1.0 + rng.uniform(-noise, noise, k)
    U = np.concatenate([[[0.0, 0.0]], np.stack([r * np.cos(ang), r * np.sin(ang)], 1)])
    T = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int64)
    return U, T


def single_charts(seed):
    """(U, T) charts for boundary_intersections."""
    rng = np.random.default_rng(seed)
    out = []
    for t in (40, 200, 900):                    # flat disks: no crossings
        P, T = synth.disk_patch(rng, t)
        out.append((P[:, :2].astype(np.float64), T.astype(np.int64)))
    for t in (200, 900, 2500):                  # boundary vertices pushed across the chart
        P, T = synth.disk_patch(rng, t)
        U = P[:, :2].astype(np.float64)
        a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]])
        b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
        n = len(U)
        bv = np.unique(a[~np.isin(b * n + a, a * n + b)])
        mv = rng.choice(bv, max(2, len(bv) // 12), replace=False)
        U[mv] = -U[mv] * rng.uniform(0.3, 1.2, (len(mv), 1))
        out.append((U, T.astype(np.int64)))
    for k, turns in ((7, 2), (40, 3), (301, 5)):   # self-winding polygons
        out.append(star_chart(rng, k, turns, 0.2))
    # exactly shared coordinates: two boundary vertices moved onto a third
    P, T = synth.disk_patch(rng, 300)
    U = P[:, :2].astype(np.float64)
    a = np.concatenate([T[:, 0], T[:, 1], T[:, 2]])
    b = np.concatenate([T[:, 1], T[:, 2], T[:, 0]])
    n = len(U)
    bv = np.unique(a[~np.isin(b * n + a, a * n + b)])
    U[bv[3]] = U[bv[len(bv) // 2]]
    U[bv[5]] = U[bv[len(bv) // 2]]
    out.append((U, T.astype(np.int64)))
    # collinear overlapping boundary edges (a chart folded onto a line)
    U = np.array([[0, 0], [2, 0], [1, 0], [3, 0], [1.5, 1.0]], np.float64)
    T = np.array([[0, 1, 4], [2, 3, 4]], np.int64)
    out.append((U, T))
    # no boundary (every half-edge has its twin) and a 2-segment boundary
    out.append((np.array([[0, 0], [1, 0], [0, 1]], np.float64), np.array([[0, 1, 2], [0, 2, 1]], np.int64)))
    # scaled tiny and huge charts
    P, T = synth.disk_patch(rng, 400)
    U = P[:, :2].astype(np.float64)
    U[rng.choice(len(U), 6, replace=False)] *= -0.7
    out.append((U * 1e-9, T.astype(np.int64)))
    out.append((U * 1e9 + 3.0, T.astype(np.int64)))
    return out


def grid_mesh(rng, nx, ny):
    s = np.arange(nx + 1, dtype=np.float64)
    X, Y = np.meshgrid(s, np.arange(ny + 1, dtype=np.float64))
    V = np.stack([X.ravel(), Y.ravel()], 1) + rng.uniform(-0.2, 0.2, ((nx + 1) * (ny + 1), 2))
    F = []
    for y in range(ny):
        for x in range(nx):
            a = y * (nx + 1) + x
            b, c, d = a + 1, a + nx + 1, a + nx + 2
            F.append([a, b, d])
            F.append([a, d, c])
    return V, np.array(F, np.int64)


def face_adjacency(F):
    owner = {}
    for f, (a, b, c) in enumerate(F):
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            owner[(u, v)] = (f, k)
    FF = -np.ones(F.shape, np.int64)
    for f, (a, b, c) in enumerate(F):
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            g = owner.get((v, u))
            if g is not None:
                FF[f, k] = g[0]
    return FF


def hier_inputs(seed, nx=36, ny=30, block=6):
    """Inputs of chart_checks: a jittered grid cut into block charts, one
    ring chart, one seam inside a chart, a few faces left out, and UVs with
    folds (pushed boundary vertices) and substituted non-finite values."""
    rng = np.random.default_rng(seed)
    V, F = grid_mesh(rng, nx, ny)
    m = len(F)
    cx = (np.arange(m) // 2) % nx
    cy = (np.arange(m) // 2) // nx
    lab = (cx // block) + (cy // block) * ((nx + block - 1) // block)
    ring = lab == lab[(2 * block + block // 2) * nx * 2 + 2 * (block + block // 2)]
    inner = ring & (cx % block >= 2) & (cx % block < block - 2) & (cy % block >= 2) & (cy % block < block - 2)
    lab = np.where(inner, lab.max() + 1, lab)
    FF = face_adjacency(F)
    faces = np.sort(rng.permutation(m)[: int(0.96 * m)])
    loc = -np.ones(m, np.int64)
    loc[faces] = np.arange(len(faces))
    ul, chart = np.unique(lab[faces], return_inverse=True)
    nchart = len(ul)
    # corner ids: one UV vertex per (chart, mesh vertex); a seam splits chart 1
    seam = (chart == 1) & (cx[faces] % block >= block // 2)
    keys = {}
    CV = np.empty((len(faces), 3), np.int64)
    for i, f in enumerate(faces):
        for k in range(3):
            key = (int(chart[i]), int(F[f, k]), bool(seam[i]))
            if key not in keys:
                keys[key] = len(keys)
            CV[i, k] = keys[key]
    nv = len(keys)
    UV = np.empty((nv, 2))
    off = rng.uniform(-3, 3, (nchart, 2))
    for (c, v, s), u in keys.items():
        UV[u] = V[v] + off[c] + (0.5 if s else 0.0)
    # folds: move a few UV vertices of some charts across their chart
    for c in rng.choice(nchart, max(2, nchart // 3), replace=False):
        ids = [u for (cc, v, s), u in keys.items() if cc == c]
        mv = rng.choice(ids, 3, replace=False)
        ctr = UV[ids].mean(0)
        UV[mv] = ctr - (UV[mv] - ctr) * 1.5
    # one chart with a non-finite UV, substituted like the reference's caller
    c = nchart - 2
    ids = [u for (cc, v, s), u in keys.items() if cc == c]
    UV[ids[0]] = 1e301
    return F, FF, faces, loc, chart, CV, UV, nchart, nv


def main(ref_root):
    sys.path.insert(0, ref_root)
    from engine import charts as rch
    from engine import hier as rhier

    out = {}
    sc = single_charts(7)
    out["bi_count"] = np.array([len(sc)])
    for i, (U, T) in enumerate(sc):
        out[f"bi_U_{i}"] = U
        out[f"bi_T_{i}"] = T
        out[f"bi_hits_{i}"] = np.array([rch.boundary_intersections(U, T, max_report=r) for r in MAX_REPORTS],
                                       np.int64)
    for s, seed in enumerate((3, 4)):
        F, FF, faces, loc, chart, CV, UV, nchart, nv = hier_inputs(seed)
        loc_in = loc.copy()
        col, chi, loops = rhier.chart_checks(F, FF, faces, loc_in, chart, CV, UV, nchart, nv)
        ba, bb = rhier.boundary_directed(F, FF, faces, loc.copy(), chart, CV)
        cc = rhier.charts_collide(CV, UV, chart, nchart, nv)
        for k, v in dict(F=F, FF=FF, faces=faces, loc=loc, chart=chart, CV=CV, UV=UV,
                         nchart=np.array([nchart]), nv=np.array([nv]), collide=col, chi=chi, loops=loops,
                         ba=ba, bb=bb, charts_collide=cc).items():
            out[f"h{s}_{k}"] = np.asarray(v)
    out["max_reports"] = np.array(MAX_REPORTS)
    path = os.path.join(HERE, "golden_segments.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: v.shape for k, v in out.items() if k.startswith("h0_") or k == "bi_count"})
    for i in range(len(sc)):
        print(i, out[f"bi_hits_{i}"])
    for s in range(2):
        print("hier", s, out[f"h{s}_collide"].astype(int), out[f"h{s}_chi"], out[f"h{s}_loops"],
              out[f"h{s}_charts_collide"].astype(int))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
