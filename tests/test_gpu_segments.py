"""Boundary self-intersection checks on the GPU (uva_boundary_hits) against
the reference's golden outputs and the oracle: charts.boundary_intersections
(count, every max_report), the batched form, hier.chart_checks and
hier.charts_collide; multi-tile charts, caps, non-finite and bad rows."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def gs():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_segments.npz"))


def _golden_charts(gs):
    return [(gs[f"bi_U_{i}"], gs[f"bi_T_{i}"], gs[f"bi_hits_{i}"]) for i in range(int(gs["bi_count"][0]))]


def test_boundary_intersections_matches_reference(cuda, gs):
    from ultimate_uv_artist_b200.engine import charts
    for i, (U, T, want) in enumerate(_golden_charts(gs)):
        got = [charts.boundary_intersections(U, T, max_report=int(r)) for r in gs["max_reports"]]
        assert got == want.tolist(), (i, got, want)


def test_boundary_intersections_batch_matches_reference(cuda, gs):
    from ultimate_uv_artist_b200.engine import charts
    ch = _golden_charts(gs)
    for k, r in enumerate(gs["max_reports"]):
        got = charts.boundary_intersections_batch([(U, T) for U, T, _ in ch], max_report=int(r))
        assert got.tolist() == [int(w[k]) for _, _, w in ch]


@pytest.mark.parametrize("s", [0, 1])
def test_chart_checks_matches_reference(cuda, gs, s):
    from ultimate_uv_artist_b200.engine import hier
    g = {k[3:]: gs[k] for k in gs.files if k.startswith(f"h{s}_")}
    nchart, nv = int(g["nchart"][0]), int(g["nv"][0])
    col, chi, loops = hier.chart_checks(g["F"], g["FF"], g["faces"], g["loc"], g["chart"], g["CV"], g["UV"],
                                        nchart, nv)
    assert np.array_equal(col, g["collide"])
    assert np.array_equal(chi, g["chi"]) and np.array_equal(loops, g["loops"])
    cc = hier.charts_collide(g["CV"], g["UV"], g["chart"], nchart, nv)
    assert np.array_equal(cc, g["charts_collide"])


def _random_charts(seed, count):
    """Star polygons (many crossings, several tiles of 128 segments) and
    disks with pushed boundary vertices."""
    from ultimate_uv_artist_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for c in range(count):
        if c % 2 == 0:
            k = int(rng.integers(3, 700))
            turns = int(rng.integers(1, 4))
            ang = np.linspace(0, 2 * np.pi * turns, k, endpoint=False) + rng.uniform(0, 0.01, k)
            r = 1 + rng.uniform(-0.3, 0.3, k)
            U = np.concatenate([[[0.0, 0.0]], np.stack([r * np.cos(ang), r * np.sin(ang)], 1)])
            T = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int64)
        else:
            P, T = synth.disk_patch(rng, int(rng.integers(20, 3000)))
            U = P[:, :2].astype(np.float64)
            mv = rng.choice(len(U), max(1, len(U) // 40), replace=False)
            U[mv] = -U[mv] * rng.uniform(0.2, 1.0, (len(mv), 1))
            T = T.astype(np.int64)
        out.append((U * rng.uniform(0.5, 50.0) + rng.uniform(-10, 10, 2), T))
    return out


def test_batch_matches_oracle_multi_tile(cuda):
    from oracle import segments as o
    from ultimate_uv_artist_b200.engine import charts
    ch = _random_charts(21, 40)
    m = [len(o.boundary_edges_oriented(T)[0]) for _, T in ch]
    assert max(m) > 3 * 128   # several tiles per chart, off-diagonal tile pairs
    for r in (1, 7, 10 ** 9):
        want = [o.boundary_intersections(U, T, r) for U, T in ch]
        got = charts.boundary_intersections_batch(ch, max_report=r)
        assert got.tolist() == want, r


def test_non_finite_and_edge_cases(cuda):
    from ultimate_uv_artist_b200 import segments
    from ultimate_uv_artist_b200.engine import charts
    U, T = _random_charts(5, 1)[0]
    bad = U.copy()
    bad[3] = np.nan
    with pytest.raises(ValueError):
        charts.boundary_intersections(bad, T)
    tiny = (np.array([[0, 0], [1, 0], [np.inf, 1]], np.float64), np.array([[0, 1, 2], [0, 2, 1]], np.int64))
    assert charts.boundary_intersections(*tiny) == 0          # fewer than 3 segments: no grid, no error
    got = charts.boundary_intersections_batch([(U, T), (bad, T), tiny])
    assert got[1] == -1 and got[2] == 0 and got[0] == charts.boundary_intersections(U, T)
    assert charts.boundary_intersections_batch([]).shape == (0,)
    # a segment row outside its chart's rows, and outside U
    seg = np.array([[0, 1], [1, 2], [2, 5]], np.int64)
    out = segments.boundary_hits(np.zeros((6, 2)), [0, 3], seg, segments.COUNT, vofs=[0, 3])
    assert out.tolist() == [-2]
    out = segments.boundary_hits(np.zeros((6, 2)), [0, 3], seg + 4, segments.ANY)
    assert out.tolist() == [-2]


def test_any_modes_extent(cuda):
    """chart_checks' extent test (1e301 substituted for non-finite UVs) and
    charts_collide's plain pair test on the same segments."""
    from oracle import segments as o
    from ultimate_uv_artist_b200 import segments
    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float64)
    seg = np.array([[0, 1], [1, 2], [2, 3], [3, 0]], np.int64)
    for UV in (sq, np.concatenate([sq[:3], [[1e301, 0.5]]])):
        want_any = o._chart_hit(UV, seg[:, 0], seg[:, 1], ext_check=True)
        want_all = o._chart_hit(UV, seg[:, 0], seg[:, 1], ext_check=False)
        assert segments.boundary_hits(UV, [0, 4], seg, segments.ANY)[0] == int(want_any)
        assert segments.boundary_hits(UV, [0, 4], seg, segments.ANY_ALL)[0] == int(want_all)


def test_batch_boundary_intersections(cuda):
    """gpu.Batch.boundary_intersections: boundary half-edges found on the
    device from the batch topology, counts at the batch's current UVs equal
    the oracle on (chart_uvs()[i], T_i), before and after the UVs change."""
    from oracle import segments as o
    from ultimate_uv_artist_b200.engine import gpu
    ch = _random_charts(33, 24)
    ch.append((np.array([[0, 0], [1, 0], [0, 1]], np.float64), np.array([[0, 1, 2], [0, 2, 1]], np.int64)))
    P = [np.concatenate([U, np.zeros((len(U), 1))], 1) for U, _ in ch]
    b = gpu.Batch([(p, T, U) for p, (U, T) in zip(P, ch)])
    for r in (1, 1000):
        want = [o.boundary_intersections(U, T, r) for U, T in ch]
        assert b.boundary_intersections(max_report=r).tolist() == want
    rng = np.random.default_rng(4)
    b.U = np.concatenate([U for U, _ in ch]) + rng.normal(0, 0.05, (b.n, 2))
    Us = b.chart_uvs()
    want = [o.boundary_intersections(Us[i], ch[i][1], 1000) for i in range(len(ch))]
    assert b.boundary_intersections().tolist() == want


@pytest.mark.parametrize("s", [0, 1])
def test_hier_topology_matches_reference(cuda, gs, s):
    from ultimate_uv_artist_b200.engine import hier
    g = {k[3:]: gs[k] for k in gs.files if k.startswith(f"h{s}_")}
    ba, bb = hier.boundary_directed(g["F"], g["FF"], g["faces"], g["loc"], g["chart"], g["CV"])
    assert np.array_equal(ba, g["ba"]) and np.array_equal(bb, g["bb"])
    chi, loops, ba2, bb2, bc = hier._boundary_topology(g["F"], g["FF"], g["faces"], g["loc"], g["chart"], g["CV"],
                                                   int(g["nchart"][0]), int(g["nv"][0]))
    assert np.array_equal(chi, g["chi"]) and np.array_equal(loops, g["loops"])
    assert len(ba2) == len(g["ba"]) and bc.min() >= 0


def test_hier_loops_mixed_components(cuda):
    """A boundary component whose vertices carry different charts: loops
    follow the reference's union order (the replayed union-find); the vertex
    charts (last naming corner) come from the device pass."""
    from oracle import segments as o
    from ultimate_uv_artist_b200.engine import hier
    # two triangles of different charts that share UV vertex ids 1 and 2
    F = np.array([[0, 1, 2], [3, 4, 5]]); FF = -np.ones((2, 3), np.int64)
    faces = np.array([0, 1]); loc = np.array([0, 1]); chart = np.array([0, 1])
    CV = np.array([[0, 1, 2], [1, 3, 2]]); UV = np.zeros((4, 2))
    want = o.chart_checks(F, FF, faces, loc, chart, CV, UV, 2, 4)
    chi, loops, *_ = hier._boundary_topology(F, FF, faces, loc, chart, CV, 2, 4)
    assert np.array_equal(chi, want[1]) and np.array_equal(loops, want[2])
