"""hier.Solver on the GPU (batch kernels: orientation, flip repair, ARAP with
the folded-chart step rule; FP64 Jacobi-PCG for the soft-pinned LSCM)
against the FP64 oracle with exact solves, and against the reference's own
float32 results (golden_hier.npz) at float32 accuracy."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def gh():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden_hier.npz"))


def _set(gh, s):
    G = {k[3:]: gh[k] for k in gh.files if k.startswith(f"s{s}_")}
    G["nv"], G["nchart"] = int(G["nv"][0]), int(G["nchart"][0])
    return G


@pytest.mark.parametrize("s", [0, 1])
def test_relax_matches_oracle_and_reference(cuda, gh, s):
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    G = _set(gh, s)
    S = hier.Solver(SimpleNamespace(V=G["V"], F=G["F"]), dev=cuda)
    U, flips, scale = S.relax(G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"], iters=6)
    Uo, fo, so, q = oh.relax(G["V"], G["F"], G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"])
    ext = np.abs(Uo).max()
    assert np.abs(U - Uo).max() <= 1e-5 * ext            # exact global steps on both sides
    assert np.array_equal(flips, fo) and np.abs(scale - so).max() <= 1e-6
    assert np.abs(U - G["U"]).max() <= 2e-4 * ext         # the reference, float32
    assert np.array_equal(flips, G["flips"])
    bA, bR = S.bad_fraction(3.0, 2.0)
    oA, oR = oh.bad_fraction(q, 3.0, 2.0)
    assert np.abs(bA - oA).max() <= 1e-3 and np.abs(bR - oR).max() <= 1e-3


@pytest.mark.parametrize("s", [0, 1])
def test_lscm_matches_oracle_and_reference(cuda, gh, s):
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    G = _set(gh, s)
    S = hier.Solver(SimpleNamespace(V=G["V"], F=G["F"]), dev=cuda)
    U = S.lscm(G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"], G["ba"], G["bb"])
    Uo = oh.lscm(G["V"], G["F"], G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"], G["ba"], G["bb"])
    ext = np.abs(Uo).max()
    assert np.abs(U - Uo).max() <= 1e-6 * ext
    assert np.abs(U - G["Ul"]).max() <= 1e-3 * ext


def test_relax_iteration_counts(cuda, gh):
    """iters 0 and 1 (repair only; the halfway repair after the only
    iteration) against the oracle."""
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    G = _set(gh, 1)
    S = hier.Solver(SimpleNamespace(V=G["V"], F=G["F"]), dev=cuda)
    for iters in (0, 1, 3):
        U, flips, _ = S.relax(G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"], iters=iters)
        Uo, fo, _, _ = oh.relax(G["V"], G["F"], G["faces"], G["CV"], G["nv"], G["chart"], G["nchart"], G["U0"],
                                iters=iters)
        assert np.abs(U - Uo).max() <= 1e-5 * np.abs(Uo).max(), iters
        assert np.array_equal(flips, fo)


def _mesh_case(nx=48, ny=40, block=16, seed=6100):
    from ultimate_uv_artist_b200 import synth
    from ultimate_uv_artist_b200.engine import hier
    V, F, FF, faces, loc, chart, CV, nv, nchart, U0 = synth.mesh_charts(seed=seed, nx=nx, ny=ny, block=block)
    ba, bb = hier.boundary_directed(F, FF, faces, loc, chart, CV)
    return V, F, faces, CV, nv, chart, nchart, U0, ba, bb


def test_lscm_device_assembly_vs_oracle_and_repeatable(cuda):
    """The device-assembled system (uva_hier_lscm) on a bumpy 48 x 40 grid
    cut into 12 charts, against the oracle's exact solve; two calls give the
    same bits (fixed entry order, no atomics in the sums)."""
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    V, F, faces, CV, nv, chart, nchart, U0, ba, bb = _mesh_case()
    S = hier.Solver(SimpleNamespace(V=V, F=F), dev=cuda)
    U = S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb)
    Uo = oh.lscm(V, F, faces, CV, nv, chart, nchart, U0, ba, bb)
    ext = np.abs(Uo).max()
    assert np.abs(U - Uo).max() <= 1e-6 * ext
    assert np.array_equal(U, S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb))


def test_lscm_permuted_ids_unused_vertices_and_empty_charts(cuda):
    """UV vertex ids shuffled across charts (the chart grouping is a sort, not
    an id range), 25 UV vertices that no face names (they keep U0, NaN
    included), faces in shuffled order, two more chart ids than charts used,
    and negative indices (counted from the end, as numpy indexing does)."""
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    V, F, faces, CV, nv, chart, nchart, U0, ba, bb = _mesh_case(nx=32, ny=32, block=16, seed=6200)
    rng = np.random.default_rng(7)
    extra = 25
    perm = rng.permutation(nv + extra)            # old id -> new id
    CVp = perm[CV]
    bap, bbp = perm[ba], perm[bb]
    U0p = rng.normal(0, 1, (nv + extra, 2))
    U0p[perm[:nv]] = U0
    U0p[perm[nv:][:3]] = np.nan
    fo = rng.permutation(len(faces))
    S = hier.Solver(SimpleNamespace(V=V, F=F), dev=cuda)
    args = (faces[fo], CVp[fo], nv + extra, chart[fo], nchart + 2, U0p, bap, bbp)
    U = S.lscm(*args)
    Uo = oh.lscm(V, F, *args)
    unused = perm[nv:]
    assert np.array_equal(U[unused], U0p[unused], equal_nan=True)
    used = perm[:nv]
    assert np.abs(U[used] - Uo[used]).max() <= 1e-6 * np.abs(Uo[used]).max()
    neg = (faces[fo] - len(F), CVp[fo] - (nv + extra), nv + extra, chart[fo], nchart + 2, U0p,
           bap - (nv + extra), bbp)
    assert np.array_equal(S.lscm(*neg), U, equal_nan=True)


def test_lscm_rejects_shared_vertices_and_bad_indices(cuda):
    from ultimate_uv_artist_b200.engine import hier
    V, F, faces, CV, nv, chart, nchart, U0, ba, bb = _mesh_case(nx=32, ny=16, block=16, seed=6300)
    S = hier.Solver(SimpleNamespace(V=V, F=F), dev=cuda)
    CVs = CV.copy()
    other = np.nonzero(chart != chart[0])[0][0]
    CVs[other, 0] = CV[0, 0]                       # a UV vertex of chart 0 in a face of another chart
    with pytest.raises(ValueError):
        S.lscm(faces, CVs, nv, chart, nchart, U0, ba, bb)
    CVb = CV.copy(); CVb[3, 1] = nv
    with pytest.raises(IndexError):
        S.lscm(faces, CVb, nv, chart, nchart, U0, ba, bb)
    chb = chart.copy(); chb[5] = nchart
    with pytest.raises(ValueError):
        S.lscm(faces, CV, nv, chb, nchart, U0, ba, bb)
    # the call after a rejected one is unaffected
    U = S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb)
    assert np.isfinite(U).all()
    assert S.lscm(faces[:0], CV[:0], 0, chart[:0], 0, U0[:0], ba[:0], bb[:0]).shape == (0, 2)


def test_lscm_degenerate_face_and_self_loop_edge(cuda):
    """A face whose UV corners repeat a vertex (its self edge folds into the
    diagonal) and a boundary edge from a vertex to itself (its two couplings
    cancel), against the oracle's COO-summed system."""
    from oracle import hier as oh
    from ultimate_uv_artist_b200.engine import hier
    V, F, faces, CV, nv, chart, nchart, U0, ba, bb = _mesh_case(nx=24, ny=16, block=8, seed=6500)
    CV = CV.copy()
    CV[5, 2] = CV[5, 1]
    ba = np.r_[ba, ba[0]]; bb = np.r_[bb, ba[0]]
    S = hier.Solver(SimpleNamespace(V=V, F=F), dev=cuda)
    U = S.lscm(faces, CV, nv, chart, nchart, U0, ba, bb)
    Uo = oh.lscm(V, F, faces, CV, nv, chart, nchart, U0, ba, bb)
    used = np.unique(CV)
    assert np.abs(U[used] - Uo[used]).max() <= 1e-6 * np.abs(Uo[used]).max()
