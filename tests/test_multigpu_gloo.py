"""Multi-GPU slab sharding, exercised with world_size 2 on CPU (gloo): the ranks' block runs
partition the planned blocks, each rank's fan window covers exactly its blocks' windows, and the
ranks agree (through an all-gather) on a layout whose concatenated slabs are the whole volume.

The data flow itself: each rank reconstructs its shard with the oracle pipeline from only the fan
views its window covers (simulated for those views alone), the slabs are all-gathered, and the
concatenation equals the single-rank reconstruction of the whole scan bit for bit."""
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


def _oracle_blocks(full, fan, f0, first, count):
    """Oracle pipeline (TEXEMU rebin, FP64 filter, column-order BP) of blocks
    [first, first + count); fan holds views from f0 on."""
    import numpy as np

    import oracle as orc

    g, ig = full.info.ctg, full.info.ig
    h = orc.ramp_taps(g.ns, g.ds)
    out = []
    for b in range(first, first + count):
        bi = full.blocks[b]
        blk = fan[bi.block_proj_start - f0: bi.block_proj_start - f0 + g.n_angle_add]
        assert blk.shape[0] == g.n_angle_add
        par = orc.rebin_fan2par(g, blk, orc.TEXEMU).astype(np.float32)
        f = orc.filter_rows_fp64(h, par).astype(np.float32)
        betas = full.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        out.append(orc.bp_par_cols(g, ig, betas, f, orc.TEXEMU))
    return np.concatenate(out, 0)


def _simulate(geo, records, v0, v1):
    import numpy as np

    import oracle as orc

    return orc.sim_project(records, geo.ns, geo.nt, geo.ds, geo.dt, np.float32(geo.central_channel),
                           np.float32((geo.nt - 1) / 2.0), geo.dso, geo.angles64(), geo.zpos64(),
                           v0, v1, 1e5, 9)


def _flow_worker(rank, world, port, geo_args, records, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from listctrecons_b200.recon import Plan
        from listctrecons_b200.scan import ScanGeometry

        geo = ScanGeometry(**geo_args)
        full = Plan(geo)
        nb = full.info.n_blocks
        first, count = shard_blocks(nb, world, rank)
        lo, hi = fan_window(full, first, count)
        fan = _simulate(geo, records, lo, hi)  # this rank's views only
        vol = torch.from_numpy(_oracle_blocks(full, fan, lo, first, count))
        cmax = -(-nb // world)
        pad = torch.zeros((cmax * 32,) + tuple(vol.shape[1:]), dtype=vol.dtype)
        pad[: vol.shape[0]] = vol
        counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(counts, torch.tensor([count], dtype=torch.int64))
        slabs = [torch.zeros_like(pad) for _ in range(world)]
        dist.all_gather(slabs, pad)
        if rank == 0:
            whole = torch.cat([s[: int(c.item()) * 32] for s, c in zip(slabs, counts)], 0)
            out.put(whole.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_reconstruct_the_single_rank_volume(small_geo):
    import numpy as np

    from listctrecons_b200.recon import Plan
    from listctrecons_b200.scan import Phantom

    geo = small_geo.with_blocks(3, cap=False)
    full = Plan(geo)
    assert full.info.n_blocks == 3  # uneven split: 2 + 1 blocks
    ph = Phantom.random(6, seed=3, fov_radius=14.0, z_lo=full.blocks[0].block_start,
                        z_hi=full.blocks[-1].block_end, semi=(2.0, 9.0))
    args = {k: getattr(geo, k) for k in geo.__dataclass_fields__}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_flow_worker, args=(r, 2, port, args, ph.records, q))
             for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    single = _oracle_blocks(full, _simulate(geo, ph.records, 0, geo.readings), 0, 0, 3)
    assert got.shape == single.shape == (3 * 32, geo.ny, geo.nx)
    assert np.abs(single).max() > 0
    np.testing.assert_array_equal(got, single)
