"""Golden fixtures of the raster atlas packer, written by the REFERENCE
implementation (Ultimate UV Artist, engine/pack.py): chart masks
(conservative raster + gutter dilation), the greedy first-fit placement of
one attempt at a fixed scale, and whole pack() runs (fine grid only below
1024 texels, coarse-to-fine above, one and three island orderings, per-chart
densities). Every run has no time budget, so the reference's result does not
depend on timing.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden_pack.py /path/to/ultimate_uv_artist
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ultimate_uv_artist_b200 import synth  # noqa: E402


def chart_set(seed, count):
    """UV charts of varied shapes: disks, elongated strips, L shapes, rings,
    in 3D units (sizes spread over 30x)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        kind = k % 4
        if kind == 0:
            P, T = synth.disk_patch(rng, int(rng.integers(30, 400)))
            U = P[:, :2].astype(np.float64)
        else:
            nx, ny = int(rng.integers(3, 12)), int(rng.integers(3, 12))
            x, y = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny))
            U = np.stack([x.ravel() * rng.uniform(1, 6), y.ravel()], 1)
            T = synth._grid_faces(nx, ny)
            c = U[T].mean(1)
            if kind == 2:     # L shape
                T = T[~((c[:, 0] > 0.5 * U[:, 0].max()) & (c[:, 1] > 0.5))]
            elif kind == 3:   # ring
                m = U.mean(0)
                T = T[np.abs(c - m).max(1) > 0.22 * np.ptp(U, 0).min()]
            used, inv = np.unique(T, return_inverse=True)
            U, T = U[used], inv.reshape(-1, 3)
        ang = rng.uniform(0, 2 * np.pi)
        R = np.array([[np.cos(ang), -np.sin(ang)], [np.sin(ang), np.cos(ang)]])
        U = (U @ R.T) * rng.uniform(0.2, 6.0) + rng.normal(0, 5, 2)
        out.append((U, np.asarray(T, np.int64)))
    return out


def main(ref_root):
    sys.path.insert(0, ref_root)
    from engine import pack

    out = {}
    charts = chart_set(61, 40)
    for k, (U, T) in enumerate(charts):
        out[f"c_U{k}"] = U
        out[f"c_T{k}"] = T
    out["c_n"] = np.array(len(charts))
    # orientation and masks of every chart at two scales (padding 0 and 2)
    for k, (U, T) in enumerate(charts):
        V = pack.orient(U)
        out[f"o_V{k}"] = V
        for tag, s, pad in (("a", 7.3, 2), ("b", 19.0, 0)):
            out[f"m{tag}_{k}"] = pack.chart_mask(V, T, s, pad)
    # one attempt at a fixed scale: placements (rotation, x, y) and occupancy
    Us = [pack.orient(U) for U, _ in charts]
    Ts = [T for _, T in charts]
    dens = np.ones(len(charts))
    tot = sum(pack._uv_area(U, T) for U, T in zip(Us, Ts))
    s_fit = 0.7 * np.sqrt(0.62 * 256 * 256 / tot)      # comfortably below the largest fitting scale
    res = pack._attempt(Us, Ts, dens, 256, 2, [0, 1, 2, 3], s_fit, "area")
    assert res is not None
    s, (placement, occ), _ = res
    out["a_place"] = np.array(placement, np.int64)
    out["a_occ"] = occ
    out["a_scale"] = np.array(s_fit)
    # a scale that does not fit (the attempt fails)
    out["a_fail_scale"] = np.array(3.0 * s_fit)
    assert pack._attempt(Us, Ts, dens, 256, 2, [0, 1, 2, 3], 3.0 * s_fit, "area") is None
    # whole runs
    runs = {
        "p1": dict(atlas=512, padding=4, grid=512, rotations=4, iters=10, orderings=("area",)),
        "p2": dict(atlas=2048, padding=8, grid=1024, rotations=4, iters=9, orderings=("area", "bbox", "height"),
                   fine_attempts=8),
        "p3": dict(atlas=1024, padding=4, grid=1024, rotations=2, iters=8, orderings=("area",), fine_attempts=4),
    }
    dens3 = np.random.default_rng(62).uniform(0.6, 1.6, len(charts))
    for name, kw in runs.items():
        density = dens3 if name == "p3" else None
        uvs, info = pack.pack(charts, density=density, time_budget=None, **kw)
        out[f"{name}_uv"] = np.concatenate(uvs)
        out[f"{name}_scale"] = np.array(info["texel_scale_grid"])
        out[f"{name}_occ"] = np.array(info["plan_occupancy"])
        if density is not None:
            out[f"{name}_dens"] = density
    path = os.path.join(HERE, "golden_pack.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
