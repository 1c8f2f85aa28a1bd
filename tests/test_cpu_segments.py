"""Boundary self-intersection checks on the CPU: the oracle against the
reference's golden outputs (tests/golden/golden_segments.npz, made by
make_golden_segments.py from the reference itself), the oracle's two forms
of the count against each other, and the host topology of engine.hier
(boundary edges, Euler characteristic, loops) against the reference."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def gs():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_segments.npz"))


def test_oracle_boundary_intersections_matches_reference(gs):
    from oracle import segments as o
    for i in range(int(gs["bi_count"][0])):
        U, T = gs[f"bi_U_{i}"], gs[f"bi_T_{i}"]
        for r, want in zip(gs["max_reports"], gs[f"bi_hits_{i}"]):
            assert o.boundary_intersections(U, T, int(r)) == want, (i, r)
            if len(U) < 400:   # the reference's own cell loops, pure Python
                assert o.boundary_intersections(U, T, int(r), loops=True) == want, (i, r)


def test_oracle_cell_loops_equal_pair_form():
    from oracle import segments as o
    rng = np.random.default_rng(12)
    for trial in range(40):
        m = int(rng.integers(3, 60))
        A = rng.uniform(-1, 1, (m, 2)); B = A + rng.normal(0, 0.6, (m, 2))
        if trial % 4 == 0:   # shared endpoints and exact duplicates
            B[1:] = np.where(rng.uniform(size=(m - 1, 1)) < 0.5, A[:-1], B[1:])
        U = np.concatenate([A, B])
        lo, cell, nx, ny = o.chart_grid(U, A, B)
        for r in (1, 4, 10 ** 6):
            assert o.seg_intersections_cells(A, B, cell, lo, nx, ny, r) == \
                o.seg_intersections_pairs(A, B, cell, lo, nx, ny, r)


@pytest.mark.parametrize("s", [0, 1])
def test_oracle_chart_checks_matches_reference(gs, s):
    from oracle import segments as o
    g = {k[3:]: gs[k] for k in gs.files if k.startswith(f"h{s}_")}
    col, chi, loops = o.chart_checks(g["F"], g["FF"], g["faces"], g["loc"], g["chart"], g["CV"], g["UV"],
                                     int(g["nchart"][0]), int(g["nv"][0]))
    assert np.array_equal(col, g["collide"]) and np.array_equal(chi, g["chi"]) and np.array_equal(loops, g["loops"])
    ba, bb = o.boundary_directed(g["F"], g["FF"], g["faces"], g["loc"], g["chart"], g["CV"])
    assert np.array_equal(ba, g["ba"]) and np.array_equal(bb, g["bb"])
    cc = o.charts_collide(g["CV"], g["UV"], g["chart"], int(g["nchart"][0]), int(g["nv"][0]))
    assert np.array_equal(cc, g["charts_collide"])
