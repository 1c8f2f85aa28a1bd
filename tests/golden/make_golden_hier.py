"""Generate the golden fixtures of hier.Solver (relax, bad_fraction, lscm)
by running the REFERENCE implementation (Ultimate UV Artist, engine/hier.py
Solver) on CPU torch with its CG run to convergence (cg_iters 3000 for
relax, iters 20000 for lscm), on a seeded mesh cut into charts.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden_hier.py /path/to/ultimate_uv_artist

The reference computes in float32 (its Solver casts frames and UVs), so the
fixtures pin the FP64 oracle to about float32 accuracy. Inputs and outputs
are stored in golden_hier.npz next to this script.
"""
from __future__ import annotations

import os
import sys
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def mesh_inputs(seed, nx=24, ny=20, block=8):
    """A bumpy grid cut into block charts with per-chart UV vertices, a
    jittered planar start with a few folds, boundary edges per chart."""
    from make_golden_segments import face_adjacency, grid_mesh
    rng = np.random.default_rng(seed)
    V2, F = grid_mesh(rng, nx, ny)
    z = 0.6 * np.sin(V2[:, 0] / 4.0) * np.cos(V2[:, 1] / 5.0) + rng.uniform(-0.05, 0.05, len(V2))
    V = np.concatenate([V2, z[:, None]], 1)
    m = len(F)
    cx = (np.arange(m) // 2) % nx
    cy = (np.arange(m) // 2) // nx
    lab = (cx // block) + (cy // block) * ((nx + block - 1) // block)
    FF = face_adjacency(F)
    faces = np.sort(rng.permutation(m)[: int(0.97 * m)])
    loc = -np.ones(m, np.int64)
    loc[faces] = np.arange(len(faces))
    _, chart = np.unique(lab[faces], return_inverse=True)
    nchart = int(chart.max()) + 1
    keys = {}
    CV = np.empty((len(faces), 3), np.int64)
    for i, f in enumerate(faces):
        for k in range(3):
            key = (int(chart[i]), int(F[f, k]))
            if key not in keys:
                keys[key] = len(keys)
            CV[i, k] = keys[key]
    nv = len(keys)
    U0 = np.empty((nv, 2))
    for (c, v), u in keys.items():
        U0[u] = V2[v] * 0.9 + rng.normal(0, 0.03, 2)
    for c in range(0, nchart, 2):   # a fold in every other chart
        ids = [u for (cc, v), u in keys.items() if cc == c]
        mv = rng.choice(ids, 2, replace=False)
        ctr = U0[ids].mean(0)
        U0[mv] = ctr + (ctr - U0[mv]) * 0.3
    return V, F, FF, faces, loc, chart, CV, nv, nchart, U0


def main(ref_root):
    sys.path.insert(0, ref_root)
    import torch
    from engine import hier as rhier
    out = {}
    for s, seed in enumerate((5, 6)):
        V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = mesh_inputs(seed)
        topo = SimpleNamespace(V=V, F=F)
        S = rhier.Solver(topo, dev=torch.device("cpu"))
        U, flips, scale = S.relax(faces, CV, nv, chart, nchart, U0, iters=6, cg_iters=3000, repair_rounds=24)
        badA, badR = S.bad_fraction(3.0, 2.0)
        ba, bb = rhier.boundary_directed(F, FF, faces, loc.copy(), chart, CV)
        Ul = S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb, iters=20000)
        for k, v in dict(V=V, F=F, FF=FF, faces=faces, loc=loc, chart=chart, CV=CV, nv=np.array([nv]),
                         nchart=np.array([nchart]), U0=U0, U=U, flips=flips, scale=scale, badA=badA, badR=badR,
                         ba=ba, bb=bb, Ul=Ul).items():
            out[f"s{s}_{k}"] = np.asarray(v)
        print("set", s, "charts", nchart, "nv", nv, "flips", flips, "scale", np.round(scale, 4))
    path = os.path.join(HERE, "golden_hier.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
