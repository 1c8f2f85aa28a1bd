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
