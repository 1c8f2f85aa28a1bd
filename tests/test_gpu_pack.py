"""GPU tests of the raster atlas packer (csrc/pack.cu through
engine/pack.py) against the reference's own outputs
(tests/golden/golden_pack.npz) and against the oracle (oracle/pack.py) on
larger seeded cases: masks bit for bit, placements and occupancy exactly,
UVs bit for bit."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = pytest.mark.gpu

RUNS = {
    "p1": dict(atlas=512, padding=4, grid=512, rotations=4, iters=10, orderings=("area",)),
    "p2": dict(atlas=2048, padding=8, grid=1024, rotations=4, iters=9, orderings=("area", "bbox", "height"),
               fine_attempts=8),
    "p3": dict(atlas=1024, padding=4, grid=1024, rotations=2, iters=8, orderings=("area",), fine_attempts=4),
}


@pytest.fixture(scope="module")
def gp():
    return dict(np.load(os.path.join(HERE, "golden", "golden_pack.npz")))


@pytest.fixture(scope="module")
def EP():
    from ultimate_uv_artist_b200.engine import pack
    return pack


def charts_of(gp):
    return [(gp[f"c_U{k}"], gp[f"c_T{k}"]) for k in range(int(gp["c_n"]))]


def test_device_masks_match_reference(gp, EP):
    n = int(gp["c_n"])
    Us = [gp[f"o_V{k}"] for k in range(n)]
    Ts = [gp[f"c_T{k}"] for k in range(n)]
    for tag, s, pad in (("a", 7.3, 2), ("b", 19.0, 0)):
        P = EP.Packer(Us, Ts, np.ones(n))
        ms = P.masks(s, pad, rot_set=(0, 1, 2, 3))
        for k in range(n):
            ref = gp[f"m{tag}_{k}"]
            assert np.array_equal(ms[k][0], ref), (tag, k)
            tiny = ref.shape[0] * ref.shape[1] < 400
            for r in (1, 2, 3):
                if tiny and r >= 2:
                    assert ms[k][r] is None
                else:
                    assert np.array_equal(ms[k][r], np.rot90(ref, r)), (tag, k, r)
    assert np.array_equal(EP.chart_mask(Us[3], Ts[3], 7.3, 2), gp["ma_3"])


def test_device_attempt_matches_reference(gp, EP):
    n = int(gp["c_n"])
    Us = [gp[f"o_V{k}"] for k in range(n)]
    Ts = [gp[f"c_T{k}"] for k in range(n)]
    P = EP.Packer(Us, Ts, np.ones(n))
    att = P.attempt(256, 2, [0, 1, 2, 3], float(gp["a_scale"]), "area")
    assert att is not None
    assert np.array_equal(np.array(att.placement), gp["a_place"])
    assert att.occupied == int(gp["a_occ"].sum())
    assert P.attempt(256, 2, [0, 1, 2, 3], float(gp["a_fail_scale"]), "area") is None
    # the page after the failed attempt is rebuilt from scratch: the same attempt again
    att2 = P.attempt(256, 2, [0, 1, 2, 3], float(gp["a_scale"]), "area")
    assert np.array_equal(np.array(att2.placement), gp["a_place"])


@pytest.mark.parametrize("name", sorted(RUNS))
def test_device_pack_runs_match_reference(gp, EP, name):
    uvs, info = EP.pack(charts_of(gp), density=gp.get(f"{name}_dens"), **RUNS[name])
    assert info["texel_scale_grid"] == float(gp[f"{name}_scale"])
    assert info["plan_occupancy"] == float(gp[f"{name}_occ"])
    assert np.array_equal(np.concatenate(uvs), gp[f"{name}_uv"])


def _random_charts(seed, count, lo=20, hi=3000):
    from ultimate_uv_artist_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        P, T = synth.disk_patch(rng, int(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        U = P[:, :2].astype(np.float64) * rng.uniform(0.2, 3.0, 2)
        ang = rng.uniform(0, 2 * np.pi)
        R = np.array([[np.cos(ang), -np.sin(ang)], [np.sin(ang), np.cos(ang)]])
        out.append((U @ R.T, np.asarray(T, np.int64)))
    return out


@pytest.mark.parametrize("ordering,rot_set,angles,G", [
    ("area", [0, 1, 2, 3], (0.0,), 1024),
    ("bbox", [0, 1], (0.0,), 700),
    ("height", [0], (0.0, 0.7853981633974483), 512),
])
def test_device_attempt_matches_oracle(EP, ordering, rot_set, angles, G):
    from oracle import pack as OP
    charts = _random_charts(7 + G, 300)
    Us = [OP.orient(U) for U, _ in charts]
    Ts = [T for _, T in charts]
    dens = np.random.default_rng(G).uniform(0.7, 1.4, len(charts))
    tot = sum(OP.uv_area(U, T) * d * d for U, T, d in zip(Us, Ts, dens))
    P = EP.Packer(Us, Ts, dens, angles)
    pad = 3
    for f in (0.55, 0.7, 0.8):
        s = f * float(np.sqrt(0.62 * G * G / tot))
        ref = OP.attempt(Us, Ts, dens, G, pad, rot_set, s, ordering, angles)
        att = P.attempt(G, pad, rot_set, s, ordering)
        assert (ref is None) == (att is None), (f, s)
        if ref is not None:
            assert att.placement == ref[1][0], f
            assert att.occupied == int(ref[1][1].sum())


def test_device_pack_many_charts_kary_search(EP):
    """1,500 islands and up take the four-probe search (pack.py:413-445)."""
    from oracle import pack as OP
    charts = _random_charts(11, 1600, lo=20, hi=200)
    kw = dict(atlas=2048, padding=4, grid=512, rotations=2, iters=6, orderings=("area",))
    uvs, info = EP.pack(charts, **kw)
    ref_uvs, ref_info = OP.pack(charts, **kw)
    assert info["texel_scale_grid"] == ref_info["texel_scale_grid"]
    assert info["plan_occupancy"] == ref_info["plan_occupancy"]
    assert np.array_equal(np.concatenate(uvs), np.concatenate(ref_uvs))


def test_device_pack_edge_cases(EP):
    # one triangle; a chart with a huge triangle (block raster path); empty list
    tri = [(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]]))]
    uvs, info = EP.pack(tri, atlas=256, padding=2, grid=256, rotations=4, iters=6)
    assert uvs[0].shape == (3, 2) and np.all((uvs[0] >= 0) & (uvs[0] <= 1))
    from oracle import pack as OP
    big = [(np.array([[0.0, 0.0], [40.0, 0.0], [0.0, 30.0], [41.0, 31.0]]), np.array([[0, 1, 2], [1, 3, 2]]))]
    big += _random_charts(5, 20)
    kw = dict(atlas=512, padding=4, grid=512, rotations=4, iters=8, orderings=("area",))
    uvs, info = EP.pack(big, **kw)
    ref_uvs, ref_info = OP.pack(big, **kw)
    assert info["texel_scale_grid"] == ref_info["texel_scale_grid"]
    assert np.array_equal(np.concatenate(uvs), np.concatenate(ref_uvs))
    uvs, info = EP.pack([], atlas=256, padding=2, grid=256, iters=3)
    assert uvs == []
    with pytest.raises(IndexError):
        EP.Packer([tri[0][0]], [np.array([[0, 1, 3]])], [1.0])


def test_device_probes_in_one_launch_match_single_attempts(EP):
    """Four attempts at different scales in one placement launch (the
    probes of a k-ary round) give what four separate attempts give."""
    from oracle import pack as OP
    charts = _random_charts(23, 400, lo=20, hi=1500)
    Us = [OP.orient(U) for U, _ in charts]
    Ts = [T for _, T in charts]
    tot = sum(OP.uv_area(U, T) for U, T in zip(Us, Ts))
    G = 512
    s0 = float(np.sqrt(0.62 * G * G / tot))
    scales = [0.6 * s0, 0.8 * s0, 0.95 * s0, 1.3 * s0]   # the last one does not fit
    P = EP.Packer(Us, Ts, np.ones(len(Us)))
    many = P.attempts_at(G, 2, [0, 1, 2, 3], scales, "bbox")
    one = [P.attempt(G, 2, [0, 1, 2, 3], s, "bbox") for s in scales]
    assert many[-1] is None and one[-1] is None
    for a, b in zip(many, one):
        assert (a is None) == (b is None)
        if a is not None:
            assert a.placement == b.placement and a.occupied == b.occupied
    assert many[0] is not None
