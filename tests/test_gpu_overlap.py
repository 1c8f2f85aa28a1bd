"""Per-chart overlap checks on the GPU (uva_overlap_raster; uva_boundary_hits
mode FIRST) against the reference's golden outputs and the oracle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def go():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_overlap.npz"))


def _pair(p):
    return [-1, -1] if p is None else list(p)


def test_overlap_checks_match_reference(cuda, go):
    from ultimate_uv_artist_b200.engine import overlapfix
    for i in range(int(go["count"][0])):
        U, T = go[f"U_{i}"], go[f"T_{i}"]
        assert np.array_equal(overlapfix.overlapping_triangles(U, T), go[f"bad_{i}"]), i
        assert np.array_equal(overlapfix.overlapping_triangles(U, T, res=64), go[f"bad64_{i}"]), i
        assert _pair(overlapfix.raster_overlap(U, T)) == go[f"pair_{i}"].tolist(), i
        assert _pair(overlapfix.collision(U, T)) == go[f"coll_{i}"].tolist(), i


def test_overlap_checks_match_oracle_random(cuda):
    """Folded disks and self-winding fans of many sizes (big triangles take
    the per-block raster path) against the oracle's serial loops."""
    from oracle import overlapfix as oo
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import overlapfix
    rng = np.random.default_rng(8)
    for trial in range(12):
        if trial % 3 == 2:
            k = int(rng.integers(5, 80))
            ang = np.linspace(0, 2 * np.pi * int(rng.integers(1, 3)), k, endpoint=False)
            U = np.concatenate([[[0.0, 0.0]], np.stack([np.cos(ang), np.sin(ang)], 1) * rng.uniform(0.6, 1.4, (k, 1))])
            T = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int64)
        else:
            P, T = synth.disk_patch(rng, int(rng.integers(20, 500)))
            U = P[:, :2].astype(np.float64)
            mv = rng.choice(len(U), max(1, len(U) // 30), replace=False)
            U[mv] = -U[mv] * rng.uniform(0.2, 1.0, (len(mv), 1))
            T = T.astype(np.int64)
        for res in (None, 40, 257):
            assert np.array_equal(overlapfix.overlapping_triangles(U, T, res), oo.overlapping_triangles(U, T, res))
            assert _pair(overlapfix.raster_overlap(U, T, res)) == _pair(oo.raster_overlap(U, T, res))
        assert _pair(overlapfix.collision(U, T)) == _pair(oo.collision(U, T))


def test_overlap_edge_cases(cuda):
    from ultimate_uv_artist_b200.engine import overlapfix
    one = (np.array([[0, 0], [1, 0], [0, 1]], np.float64), np.array([[0, 1, 2]], np.int64))
    assert not overlapfix.overlapping_triangles(*one).any() and overlapfix.raster_overlap(*one) is None
    flat = (np.zeros((4, 2)), np.array([[0, 1, 2], [1, 3, 2]], np.int64))   # zero extent
    assert not overlapfix.overlapping_triangles(*flat).any() and overlapfix.raster_overlap(*flat) is None
    U = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [np.nan, 0]], np.float64)
    T = np.array([[0, 1, 2], [1, 3, 2], [2, 3, 4]], np.int64)
    assert not overlapfix.overlapping_triangles(U, T).any()   # non-finite extent: nothing marked
    with pytest.raises(ValueError):
        overlapfix.collision(U, T)
