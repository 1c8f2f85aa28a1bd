"""Per-chart overlap checks on the CPU: the oracle (oracle/overlapfix.py,
serial loops in the reference's order) against the reference's own outputs
(tests/golden/golden_overlap.npz, made by make_golden_overlap.py)."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def go():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_overlap.npz"))


def _pair(p):
    return [-1, -1] if p is None else list(p)


def test_oracle_overlap_checks_match_reference(go):
    from oracle import overlapfix as oo
    for i in range(int(go["count"][0])):
        U, T = go[f"U_{i}"], go[f"T_{i}"]
        if len(T) <= 700:   # pure-Python rasters: the small charts
            assert np.array_equal(oo.overlapping_triangles(U, T), go[f"bad_{i}"]), i
            assert _pair(oo.raster_overlap(U, T)) == go[f"pair_{i}"].tolist(), i
        assert np.array_equal(oo.overlapping_triangles(U, T, res=64), go[f"bad64_{i}"]), i
        assert _pair(oo.collision(U, T)) == go[f"coll_{i}"].tolist(), i
