"""Generate the golden fixtures of the per-chart overlap checks by running the
REFERENCE implementation (Ultimate UV Artist, engine/overlapfix.py:
overlapping_triangles, raster_overlap, collision) on small seeded charts.

    NUMBA_CACHE_DIR=/tmp/nb python tests/golden/make_golden_overlap.py /path/to/ultimate_uv_artist

Inputs and outputs are stored in golden_overlap.npz next to this script.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def charts(seed):
    from make_golden_segments import single_charts, star_chart
    rng = np.random.default_rng(seed)
    out = [c for c in single_charts(seed) if len(c[1]) >= 1]
    for k, turns in ((12, 1), (60, 2)):
        out.append(star_chart(rng, k, turns, 0.1))
    return out


def main(ref_root):
    sys.path.insert(0, ref_root)
    from engine import overlapfix as rof
    out = {}
    ch = charts(17)
    out["count"] = np.array([len(ch)])
    for i, (U, T) in enumerate(ch):
        out[f"U_{i}"] = U
        out[f"T_{i}"] = T
        out[f"bad_{i}"] = rof.overlapping_triangles(U, T)
        out[f"bad64_{i}"] = rof.overlapping_triangles(U, T, res=64)
        p = rof.raster_overlap(U, T)
        out[f"pair_{i}"] = np.array([-1, -1] if p is None else list(p), np.int64)
        try:
            c = rof.collision(U, T)
        except Exception:  # noqa: BLE001 - the reference raises on some inputs
            c = (-9, -9)
        out[f"coll_{i}"] = np.array([-1, -1] if c is None else list(c), np.int64)
        print(i, len(T), int(out[f"bad_{i}"].sum()), out[f"pair_{i}"], out[f"coll_{i}"])
    path = os.path.join(HERE, "golden_overlap.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UVA_REFERENCE", ""))
