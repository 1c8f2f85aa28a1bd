"""hier.Solver's batch layout (host numpy, no GPU): charts as islands in
chart order, each chart's UV vertices in id order, the faces grouped by chart
in input order, positions from the mesh vertex of a corner naming each UV
vertex; checked against a loop restatement on shuffled ids."""
import numpy as np
import pytest


def _loop_layout(V, F, faces, CV, nv, chart, nchart):
    vchart = {}
    vmesh = {}
    for f in range(len(faces)):
        for k in range(3):
            vchart[int(CV[f, k])] = int(chart[f])
            vmesh[int(CV[f, k])] = int(F[faces[f], k])
    order = [v for c in range(nchart) for v in sorted(u for u, cc in vchart.items() if cc == c)]
    newid = {v: i for i, v in enumerate(order)}
    vofs = np.cumsum([0] + [sum(1 for cc in vchart.values() if cc == c) for c in range(nchart)])
    forder = [f for c in range(nchart) for f in range(len(faces)) if chart[f] == c]
    tofs = np.cumsum([0] + [int((chart == c).sum()) for c in range(nchart)])
    T_local = np.array([[newid[int(CV[f, k])] - vofs[chart[f]] for k in range(3)] for f in forder])
    P = np.array([V[vmesh[v]] for v in order])
    return np.array(order), P, T_local, vofs, tofs, np.array(forder)


def test_layout_matches_loop_restatement_on_shuffled_ids():
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import hier
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts(seed=6400, nx=12, ny=10, block=5)
    rng = np.random.default_rng(11)
    perm = rng.permutation(nv + 4)
    fo = rng.permutation(len(faces))
    args = (faces[fo], perm[CV][fo], nv + 4, chart[fo], nchart + 1)
    S = hier.Solver.__new__(hier.Solver)   # the layout needs no device
    S.V, S.F = np.asarray(V, np.float64), np.asarray(F, np.int64)
    got = S._layout(*args)
    want = _loop_layout(S.V, S.F, *args)
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w))


def test_layout_rejects_a_vertex_of_two_charts():
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import hier
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts(seed=6401, nx=10, ny=10, block=5)
    CVs = CV.copy()
    other = np.nonzero(chart != chart[0])[0][0]
    CVs[other, 1] = CV[0, 0]
    S = hier.Solver.__new__(hier.Solver)
    S.V, S.F = np.asarray(V, np.float64), np.asarray(F, np.int64)
    with pytest.raises(ValueError):
        S._layout(faces, CVs, nv, chart, nchart)
