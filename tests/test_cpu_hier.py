"""hier.Solver on the CPU: the FP64 oracle (oracle/hier.py, exact solves)
against the reference's Solver run to convergence on CPU torch
(tests/golden/golden_hier.npz, made by make_golden_hier.py). The reference
computes in float32, so the pins hold at float32 accuracy."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def gh():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_hier.npz"))


def _set(gh, s):
    G = {k[3:]: gh[k] for k in gh.files if k.startswith(f"s{s}_")}
    G["nv"], G["nchart"] = int(G["nv"][0]), int(G["nchart"][0])
    return G


@pytest.mark.parametrize("s", [0, 1])
def test_oracle_relax_matches_reference(gh, s):
    from oracle import hier as oh
    G = _set(gh, s)
    U, flips, scale, q = oh.relax(G["V"], G["F"], G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"])
    assert np.abs(U - G["U"]).max() <= 2e-4 * np.abs(G["U"]).max()
    assert np.array_equal(flips, G["flips"])
    assert np.abs(scale - G["scale"]).max() <= 1e-4
    bA, bR = oh.bad_fraction(q, 3.0, 2.0)
    assert np.abs(bA - G["badA"]).max() <= 1e-3 and np.abs(bR - G["badR"]).max() <= 1e-3


@pytest.mark.parametrize("s", [0, 1])
def test_oracle_lscm_matches_reference(gh, s):
    from oracle import hier as oh
    G = _set(gh, s)
    Ul = oh.lscm(G["V"], G["F"], G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"], G["ba"], G["bb"])
    assert np.abs(Ul - G["Ul"]).max() <= 1e-3 * np.abs(G["Ul"]).max()


def test_solver_layout_groups_charts(gh):
    """The batch layout of Solver.relax: islands in chart order, each chart's
    UV vertices in id order, local triangles, positions from the mesh."""
    from ultimate_uv_artist_b200.engine import hier
    G = _set(gh, 0)
    S = hier.Solver.__new__(hier.Solver)
    S.V, S.F = G["V"], G["F"]
    order, P, T_local, vofs, tofs, forder = S._layout(G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"])
    assert len(order) == len(np.unique(G["CV"])) and (np.diff(vofs) > 0).all()
    for c in range(G["nchart"]):
        vs = order[vofs[c]:vofs[c + 1]]
        assert (np.diff(vs) > 0).all()
        fs = forder[tofs[c]:tofs[c + 1]]
        assert (G["chart"][fs] == c).all()
        assert np.array_equal(vs[T_local[tofs[c]:tofs[c + 1]]], G["CV"][fs])
    newid = np.empty(G["nv"], np.int64)
    newid[order] = np.arange(len(order))
    assert np.array_equal(P[newid[G["CV"][:, 0]]], G["V"][G["F"][G["faces"], 0]])
    bad = G["CV"].copy()
    bad[0, 0] = G["CV"][np.nonzero(G["chart"] != G["chart"][0])[0][0], 0]   # a vertex of another chart
    with pytest.raises(ValueError):
        S._layout(G["faces"], bad, G["nv"], G["chart"], G["nchart"])


def test_mesh_charts_workload_is_consistent():
    """synth.mesh_charts (the bench's hier.Solver workload): face adjacency
    across each corner edge, chart-private UV vertices, and the oracle's
    chart topology (one boundary loop, disk charts) on a small instance."""
    from oracle import segments as OS
    from ultimate_uv_artist_b200 import synth
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts(nx=24, ny=16, block=8)
    owner = {}
    for f, (a, b, c) in enumerate(F.tolist()):
        for u, v in ((a, b), (b, c), (c, a)):
            owner[(u, v)] = f
    for f, (a, b, c) in enumerate(F.tolist()):
        for k, (u, v) in enumerate(((a, b), (b, c), (c, a))):
            assert FF[f, k] == owner.get((v, u), -1)
    vch = -np.ones(nv, np.int64)
    for i in range(len(CV)):
        for v in CV[i]:
            assert vch[v] in (-1, chart[i])
            vch[v] = chart[i]
    assert nchart == 6 and U0.shape == (nv, 2) and np.isfinite(U0).all()
    col, chi, loops = OS.chart_checks(F, FF, faces, loc, chart, CV, U0, nchart, nv)
    assert (chi == 1).all() and (loops == 1).all()
