"""CPU tests of the raster atlas packer's oracle against the reference's own
outputs (tests/golden/golden_pack.npz, written by make_golden_pack.py from
engine/pack.py): orientation, chart masks at two scales and paddings, the
first-fit placement of one attempt, a failing attempt and three whole
pack() runs (fine grid only, coarse-to-fine with three orderings,
per-chart densities with two rotations). Also the host-side sizing the
device packer uses. No GPU needed."""
import os

import numpy as np
import pytest

from oracle import pack as OP

HERE = os.path.dirname(os.path.abspath(__file__))
RUNS = {
    "p1": dict(atlas=512, padding=4, grid=512, rotations=4, iters=10, orderings=("area",)),
    "p2": dict(atlas=2048, padding=8, grid=1024, rotations=4, iters=9, orderings=("area", "bbox", "height"),
               fine_attempts=8),
    "p3": dict(atlas=1024, padding=4, grid=1024, rotations=2, iters=8, orderings=("area",), fine_attempts=4),
}


@pytest.fixture(scope="module")
def gp():
    return dict(np.load(os.path.join(HERE, "golden", "golden_pack.npz")))


def charts_of(gp):
    return [(gp[f"c_U{k}"], gp[f"c_T{k}"]) for k in range(int(gp["c_n"]))]


def test_oracle_orient_and_masks_match_reference(gp):
    for k, (U, T) in enumerate(charts_of(gp)):
        assert np.array_equal(OP.orient(U), gp[f"o_V{k}"]), k
        assert np.array_equal(OP.chart_mask(gp[f"o_V{k}"], T, 7.3, 2), gp[f"ma_{k}"]), k
        assert np.array_equal(OP.chart_mask(gp[f"o_V{k}"], T, 19.0, 0), gp[f"mb_{k}"]), k


def test_oracle_intervals_round_trip(gp):
    for k in range(6):
        m = np.rot90(gp[f"ma_{k}"], k % 4)
        ptr, a, b, need = OP.intervals(m)
        back = np.zeros_like(m)
        for j in range(m.shape[0]):
            for q in range(ptr[j], ptr[j + 1]):
                back[j, a[q]:b[q] + 1] = 1
            runs = b[ptr[j]:ptr[j + 1]] - a[ptr[j]:ptr[j + 1]] + 1
            assert need[j] == (runs.max() if len(runs) else 0)
        assert np.array_equal(back, m)


def test_oracle_attempt_matches_reference(gp):
    n = int(gp["c_n"])
    Us = [gp[f"o_V{k}"] for k in range(n)]
    Ts = [gp[f"c_T{k}"] for k in range(n)]
    r = OP.attempt(Us, Ts, np.ones(n), 256, 2, [0, 1, 2, 3], float(gp["a_scale"]), "area")
    assert r is not None
    placement, occ = r[1]
    assert np.array_equal(np.array(placement), gp["a_place"])
    assert np.array_equal(occ, gp["a_occ"])
    assert OP.attempt(Us, Ts, np.ones(n), 256, 2, [0, 1, 2, 3], float(gp["a_fail_scale"]), "area") is None


@pytest.mark.parametrize("name", sorted(RUNS))
def test_oracle_pack_runs_match_reference(gp, name):
    dens = gp.get(f"{name}_dens")
    uvs, info = OP.pack(charts_of(gp), density=dens, **RUNS[name])
    assert info["texel_scale_grid"] == float(gp[f"{name}_scale"])
    assert info["plan_occupancy"] == float(gp[f"{name}_occ"])
    assert np.array_equal(np.concatenate(uvs), gp[f"{name}_uv"])


def test_mask_size_from_vertex_maxima(gp):
    """The device packer sizes each mask from the chart's largest coordinates
    (rounding is monotone): the sizes equal the reference's masks'."""
    from ultimate_uv_artist_b200.engine import pack as EP
    for k in range(int(gp["c_n"])):
        V = gp[f"o_V{k}"]
        for tag, s, pad in (("a", 7.3, 2), ("b", 19.0, 0)):
            h, w = EP.mask_shape(V.max(0), s, pad)
            assert (h, w) == gp[f"m{tag}_{k}"].shape
