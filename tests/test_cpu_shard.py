"""Multi-rank host logic (islands sharded across ranks, no data-path
collective), run as two gloo processes on the CPU: the partition every rank
computes on its own, the gather of per-island results in island order, and
the max / sum reduction of step timings that bench.py reports."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from ultimate_uv_artist_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(7)
        sizes = np.exp(rng.uniform(np.log(20), np.log(20000), 50)).astype(int)
        charts = [(np.zeros((s // 2 + 3, 3)), np.zeros((s, 3), np.int64)) for s in sizes]
        idx, mine = shard.shard_charts(charts, rank, world)
        # a stand-in per-island result: the island index in every UV row
        local = [np.full((len(ch[0]), 2), float(i)) for i, ch in zip(idx, mine)]
        allu = shard.gather_chart_uvs(local, idx, len(charts))
        ok_gather = all(u.shape == (len(charts[i][0]), 2) and (u == i).all() for i, u in enumerate(allu))
        on0 = shard.gather_chart_uvs(local, idx, len(charts), dst=0)
        ok_dst = (on0 is not None) == (rank == 0)
        load = float(sum(len(ch[1]) for ch in mine))
        ms, units = shard.reduce_step(10.0 + rank, load)
        q.put((rank, idx.tolist(), load, ok_gather, ok_dst, ms, units, int(sizes.sum())))
    finally:
        dist.destroy_process_group()


def test_lpt_partition_properties():
    from ultimate_uv_artist_b200 import shard
    costs = [5, 9, 1, 9, 3, 7, 7, 2]
    parts = shard.lpt_partition(costs, 3)
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert [p.tolist() for p in parts] == [p.tolist() for p in shard.lpt_partition(costs, 3)]
    assert [p.tolist() for p in shard.lpt_partition(costs, 1)] == [list(range(len(costs)))]
    with pytest.raises(ValueError):
        shard.lpt_partition(costs, 0)


def test_two_gloo_ranks_shard_gather_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    idx0, idx1 = set(res[0][1]), set(res[1][1])
    assert not (idx0 & idx1) and len(idx0 | idx1) == 50      # every island on exactly one rank
    total = res[0][7]
    for r in res:
        assert r[3] and r[4]                                  # gather in island order; dst-only gather
        assert r[5] == 11.0 and r[6] == total                 # max of step times, sum of units
    assert abs(res[0][2] - res[1][2]) <= 20000                # LPT balance within one island


def _val_worker(rank, world, port, q):
    """One validation shard: the oracle's band of the overlap scan (the
    per-rank compute stands in for the device), the product's all-reduce of
    the overlap bits and pair counts, compared with the unsharded scan."""
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import validate as OV
    from ultimate_uv_artist_b200 import shard, synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        V, F, UV, _ = synth.validation_atlas(seed=41, islands=120, tris_per_island=60, atlas=512, padding=4,
                                             overlap_rate=5e-3, fold_rate=2e-3, mirrored=1, outside=3)
        U = np.asarray(UV, np.float32).astype(np.float64)
        _, _, ex = OV.validate_uvs(V, F, UV, atlas=512, padding=4, gutter=False, count_pairs=False)
        skip, G = ex["skip"], int(np.clip(np.sqrt(len(F)) / 2, 64, 4096))
        ok = True
        for strict in (False, True):
            full, nfull = OV.overlaps_c(U, F, skip, G, 0.0 if strict else 1e-6, strict=strict)
            part, npart = OV.overlaps_c(U, F, skip, G, 0.0 if strict else 1e-6, strict=strict,
                                        band=shard.band_rows(G, rank, world))
            merged = shard.allreduce_max(torch.from_numpy(part.astype(np.uint8)), None).numpy().astype(bool)
            tested = int(shard.allreduce_sum(torch.tensor([npart], dtype=torch.int64), None)[0])
            ok &= bool(np.array_equal(merged, full)) and tested == nfull and bool(full.any())
        q.put((rank, ok, shard.rank_world(dist.group.WORLD)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_validation_bands():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_val_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [True, True]
    assert [r[2] for r in res] == [(0, 2), (1, 2)]


def test_band_rows_cover_the_grid_once():
    from ultimate_uv_artist_b200 import shard
    for G in (64, 100, 4096):
        for world in (1, 2, 3, 8):
            rows = [shard.band_rows(G, r, world) for r in range(world)]
            assert rows[0][0] == 0 and rows[-1][1] == G
            assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
    assert shard.rank_world(None) == (0, 1)
