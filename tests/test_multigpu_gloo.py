"""Multi-GPU slab sharding, exercised with world_size 2 on CPU (gloo): the ranks' block runs
partition the planned blocks, each rank's fan window covers exactly its blocks' windows, and the
ranks agree (through an all-gather) on a layout whose concatenated slabs are the whole volume."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from listctrecons_b200.shard import fan_window, shard_blocks


def test_shard_blocks_partition():
    for n in (1, 7, 16, 93):
        for world in (1, 2, 3, 8):
            if world > n:
                continue
            runs = [shard_blocks(n, world, r) for r in range(world)]
            covered = [b for f, c in runs for b in range(f, f + c)]
            assert covered == list(range(n))
    assert shard_blocks(16, 2, 1, per_rank=8) == (8, 8)
    with pytest.raises(ValueError):
        shard_blocks(16, 4, 0, per_rank=8)


def _worker(rank, world, port, geo_args, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from listctrecons_b200.recon import Plan
        from listctrecons_b200.scan import ScanGeometry

        geo = ScanGeometry(**geo_args)
        full = Plan(geo)
        first, count = shard_blocks(full.info.n_blocks, world, rank)
        p = geo.scan_params()
        p.first_block, p.max_blocks = first, count
        mine = Plan(params=p, angles32=geo.angles32(), zpos32=geo.zpos32())
        assert mine.info.first_block == first and mine.info.n_blocks_run == count
        lo, hi = fan_window(full, first, count)
        t = torch.tensor([first, count, lo, hi], dtype=torch.int64)
        got = [torch.zeros(4, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(got, t)
        if rank == 0:
            out.put([g.tolist() for g in got])
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_with_gloo(small_geo):
    from listctrecons_b200.recon import Plan

    geo = small_geo.with_blocks(5, cap=False)
    args = {k: getattr(geo, k) for k in geo.__dataclass_fields__}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, args, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    full = Plan(geo)
    (f0, c0, lo0, hi0), (f1, c1, lo1, hi1) = res
    assert f0 == 0 and f1 == c0 and c0 + c1 == full.info.n_blocks
    for f, c, lo, hi in res:
        starts = [full.blocks[b].block_proj_start for b in range(f, f + c)]
        assert lo == min(starts) and hi == max(starts) + full.info.ctg.n_angle_add
        assert 0 <= lo and hi <= geo.readings
