"""GPU validation kernels against the reference (golden fixtures) and the
oracle. Verdicts must match bit for bit: every report count, the problem mask,
the overlap and strict-overlap masks and the island partition."""
import numpy as np
import pytest

from oracle import validate as OV

pytestmark = pytest.mark.gpu

KEYS = ["non_finite_uv", "uv_outside_unit_square", "degenerate_uv_triangles", "sub_float32_slivers",
        "flipped_triangles", "mirrored_islands", "islands", "overlapping_triangles_exact", "float32_contacts",
        "islands_with_overlap", "min_gutter_texels", "gutter_ok", "valid"]


def _device_masks(V, F, UV):
    from ultimate_uv_artist_b200.engine import validate as GV
    dv = GV.DeviceValidation(np.asarray(V, np.float64), np.asarray(F, np.int32), np.asarray(UV, np.float32)).run()
    fl = dv.flags()
    return fl, dv.labels[:len(F)].cpu().numpy(), dv.host_counts()


def _compare(rep, ref, keys=KEYS):
    for k in keys:
        if k in ref:
            assert k in rep, k
            a, b = float(rep[k]), float(ref[k])
            assert a == b or (np.isnan(a) and np.isnan(b)), (k, rep[k], ref[k])


@pytest.mark.parametrize("prefix", ["v", "w"])
def test_report_matches_reference_golden(golden, cuda, prefix):
    from ultimate_uv_artist_b200.engine import validate as GV
    V, F, UV = golden[f"{prefix}_V"], golden[f"{prefix}_F"], golden[f"{prefix}_UV"]
    rep, problems = GV.validate_uvs(V, F, UV, atlas=512, padding=4)
    ref = dict(zip(golden[f"{prefix}_rep_keys"].tolist(), golden[f"{prefix}_rep_vals"].tolist()))
    _compare(rep, ref)
    assert np.array_equal(problems, golden[f"{prefix}_problems"])
    fl, lab, _ = _device_masks(V, F, UV)
    assert OV.same_partition(lab, golden[f"{prefix}_isl"])
    if prefix == "v":
        assert np.array_equal((fl & 16) != 0, golden["v_ov"])
        assert np.array_equal((fl & 32) != 0, golden["v_ovs"])


def test_chart_overlaps_matches_reference(golden, cuda):
    from ultimate_uv_artist_b200.engine import validate as GV
    got = GV.chart_overlaps(golden["v_cU"], golden["v_cF"])
    assert np.array_equal(got, golden["v_cov"])
    # a chart folded onto itself: must overlap, same flags as the oracle
    U = golden["v_cU"].copy()
    T = golden["v_cF"]
    U[T[3, 0]] = U[T[40, 2]] + (U[T[40, 0]] - U[T[40, 2]]) * 0.5
    assert np.array_equal(GV.chart_overlaps(U, T), OV.chart_overlaps(U, T))


def _full_compare(V, F, UV, atlas, padding):
    from ultimate_uv_artist_b200.engine import validate as GV
    rep, problems = GV.validate_uvs(V, F, UV, atlas=atlas, padding=padding)
    ref, rprob, ex = OV.validate_uvs(V, F, UV, atlas=atlas, padding=padding)
    _compare(rep, ref)
    assert np.array_equal(problems, rprob)
    fl, lab, cnt = _device_masks(V, F, UV)
    assert np.array_equal((fl & 16) != 0, ex["ov"])
    assert np.array_equal((fl & 32) != 0, ex["ov_strict"])
    assert np.array_equal((fl & 8) != 0, ex["flipped"])
    assert OV.same_partition(lab, ex["islands"])
    assert int(cnt[10]) == ex["pairs"], (int(cnt[10]), ex["pairs"])
    return rep


def test_validation_atlas_medium_bit_exact(cuda):
    from ultimate_uv_artist_b200 import synth
    V, F, UV, _ = synth.validation_atlas(seed=3100, islands=800, tris_per_island=200, atlas=2048, padding=4,
                                         overlap_rate=3e-4, fold_rate=5e-5, mirrored=3, outside=20)
    rep = _full_compare(V, F, UV, 2048, 4)
    assert rep["overlapping_triangles_exact"] > 0 and rep["flipped_triangles"] > 0


def test_validation_atlas_full_size_bit_exact(cuda):
    """The 1M-triangle, 5,000-island atlas (4096, padding 4) with injected
    overlaps, folds, mirrored islands and out-of-range vertices."""
    from ultimate_uv_artist_b200 import synth
    V, F, UV, info = synth.validation_atlas(seed=3000)
    rep = _full_compare(V, F, UV, 4096, 4)
    assert rep["mirrored_islands"] >= 3 and rep["uv_outside_unit_square"] == 20


def test_clean_atlas_gutter_exact(cuda):
    from ultimate_uv_artist_b200 import synth
    V, F, UV, _ = synth.validation_atlas(seed=3200, islands=300, tris_per_island=50, atlas=1024, padding=6,
                                         overlap_rate=0.0, fold_rate=0.0, mirrored=0, outside=0)
    rep = _full_compare(V, F, UV, 1024, 4)
    assert rep["min_gutter_texels"] > 0


def test_edge_cases(cuda):
    """Empty input, NaN and out-of-range UVs, zero-area and duplicated triangles."""
    from ultimate_uv_artist_b200.engine import validate as GV
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [2, 2, 0]], float)
    UV = np.array([[0.1, 0.1], [0.6, 0.1], [0.1, 0.6], [0.6, 0.6], [0.3, 0.3]], float)
    F = np.array([[0, 1, 2], [1, 3, 2], [0, 1, 2], [0, 4, 3]])       # duplicate + overlapping
    for uv in (UV, np.r_[UV[:4], [[np.nan, 0.2]]], np.r_[UV[:4], [[1.5, -0.2]]]):
        rep, prob = GV.validate_uvs(V, F, uv, atlas=64, padding=2)
        ref, rprob, _ = OV.validate_uvs(V, F, uv, atlas=64, padding=2)
        _compare(rep, ref)
        assert np.array_equal(prob, rprob)
    # zero 3D area and zero UV area triangles
    V2 = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0]], float)
    F2 = np.array([[0, 1, 2], [0, 1, 3]])
    UV2 = np.array([[0.1, 0.1], [0.2, 0.1], [0.3, 0.1], [0.1, 0.3]])
    rep, prob = GV.validate_uvs(V2, F2, UV2, atlas=64)
    ref, rprob, _ = OV.validate_uvs(V2, F2, UV2, atlas=64)
    _compare(rep, ref)
    # no triangles
    rep, prob = GV.validate_uvs(V2, np.zeros((0, 3), np.int64), UV2, atlas=64, gutter=False)
    assert rep["islands"] == 0 and rep["valid"] and len(prob) == 0


def test_validation_shards_merge_to_the_whole(cuda):
    """Sharded validation on one GPU, the shards one after another: each
    shard's overlap bits equal the oracle's scan of the same band of cell
    rows, the bits OR'd together and the pair counts summed give the
    unsharded flags, and uva_validate_finish the unsharded counts; with a
    process group (gloo, one rank) validate_uvs gives the whole report."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    from ultimate_uv_artist_b200 import shard, synth
    from ultimate_uv_artist_b200.engine import validate as GV
    V, F, UV, _ = synth.validation_atlas(seed=3100, islands=800, tris_per_island=200, atlas=2048, padding=4,
                                         overlap_rate=3e-4, fold_rate=5e-5, mirrored=3, outside=20)
    F32 = F.astype(np.int32)
    whole = GV.DeviceValidation(V, F32, UV).run()
    w_flags, w_counts = whole.flags(), whole.host_counts()
    _, _, ex = OV.validate_uvs(V, F, UV, atlas=2048, padding=4, gutter=False, count_pairs=False)
    U = np.asarray(UV, np.float32).astype(np.float64)
    G = int(np.clip(np.sqrt(len(F)) / 2, 64, 4096))
    world = 3
    parts = [GV.DeviceValidation(V, F32, UV, shard=r, nshards=world).run() for r in range(world)]
    bits = np.zeros(len(F), np.uint8)
    pairs = 0
    for r, dv in enumerate(parts):
        fl = dv.flags()
        band = shard.band_rows(G, r, world)
        ov, _ = OV.overlaps_c(U, F, ex["skip"], G, 1e-6, band=band)
        ovs, _ = OV.overlaps_c(U, F, ex["skip"], G, 0.0, strict=True, band=band)
        assert np.array_equal((fl & 16) != 0, ov) and np.array_equal((fl & 32) != 0, ovs), r
        assert np.array_equal(fl & 15, w_flags & 15), r     # the band leaves the other bits alone
        bits |= fl & 48
        pairs += int(dv.host_counts()[GV.VC_PAIRS])
    head = parts[0]
    head.tflags[:len(F)] = torch.from_numpy((head.flags() & 207) | bits).to(head.tflags.device)
    head.counts[GV.VC_PAIRS] = pairs
    head.finish()
    assert np.array_equal(head.flags(), w_flags)
    assert np.array_equal(head.host_counts(), w_counts)
    # the process-group path (one gloo rank: the merge is the identity, finish recounts)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rep_g, prob_g = GV.validate_uvs(V, F, UV, atlas=2048, padding=4, group=dist.group.WORLD)
        dv = GV.DeviceValidation(V, F32, UV).run().merge(dist.group.WORLD)
        assert np.array_equal(dv.host_counts(), w_counts)
    finally:
        dist.destroy_process_group()
    rep, prob = GV.validate_uvs(V, F, UV, atlas=2048, padding=4)
    assert rep_g == rep and np.array_equal(prob_g, prob)
