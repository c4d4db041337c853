"""Batched reconstruction (lct_batch: one graph launch per stage, one persistent work-list
backprojection over every scan) and the backprojection autotuner.  Bar: each scan's batch volume
is bit-identical to its own lct_recon run with the same options -- with one requested thread
shape, and with each scan's own default shape (several work lists); the autotuned run equals the
default one in TEX8 mode, whose arithmetic per slice does not depend on the thread shape."""
import numpy as np
import pytest

from listctrecons_b200 import capi
from listctrecons_b200.recon import Batch, Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu

pytestmark = pytest.mark.gpu

GEOS = [
    dict(ns=96, nt=8, ds=1.0, dt=1.0, npt=120, pitch=1.0, nx=32, ny=32, dx=1.0, dz=1.0, blocks=2),
    dict(ns=80, nt=16, ds=0.8, dt=0.6, npt=100, pitch=0.7, nx=24, ny=40, dx=0.9, dz=0.5, blocks=1),
    dict(ns=112, nt=8, ds=0.9, dt=1.1, npt=150, pitch=1.3, nx=40, ny=40, dx=0.8, dz=1.2, blocks=3),
]


@pytest.fixture(scope="module")
def scans(cuda):
    out = []
    for i, d in enumerate(GEOS):
        d = dict(d)
        nb = d.pop("blocks")
        geo = ScanGeometry(**d).with_blocks(nb)
        p = Plan(geo)
        lo = min(p.blocks[0].block_start, p.blocks[nb - 1].block_end)
        hi = max(p.blocks[0].block_start, p.blocks[nb - 1].block_end)
        ph = Phantom.random(5, seed=40 + i, fov_radius=0.45 * geo.nx * geo.dx, z_lo=lo, z_hi=hi,
                            semi=(2.0, 9.0))
        out.append((geo, p, simulate_gpu(geo, ph, i0=1e5, seed=11 + i)))
    return out


@pytest.mark.parametrize("interp,bp_nz", [(capi.INTERP_EXACT, 8), (capi.INTERP_TEX8, 8),
                                          (capi.INTERP_EXACT, 0)])
def test_batch_equals_single_scan_runs(scans, interp, bp_nz):
    """bp_nz 0: each scan keeps its default shape (4 or 8 slices per thread for these three
    scans), so the backprojection graph holds one work list per shape."""
    import torch

    plans = [p for _, p, _ in scans]
    b = Batch(plans, interp=interp, filter_mode=capi.FILTER_BF16X6, bp_nz=bp_nz)
    imgs = b.run([f for _, _, f in scans])
    torch.cuda.synchronize()
    for (geo, p, fan), img in zip(scans, imgs):
        single = Reconstruction(p, interp=interp, filter_mode=capi.FILTER_BF16X6,
                                bp_nz=bp_nz).run(fan)
        assert torch.equal(img, single)
    # host buffers in and out give the same volumes
    hf = [f.cpu().pin_memory() for _, _, f in scans]
    hi = [torch.empty(sh, dtype=torch.float32).pin_memory() for sh in b.image_shapes]
    b.run(hf, hi)
    for a, c in zip(hi, imgs):
        assert np.array_equal(a.numpy(), c.cpu().numpy())
    t = b.last_times()
    assert t["backproject"] > 0 and b.stats().voxel_updates > 0


def test_autotune_keeps_results(scans):
    import torch

    _, p, fan = scans[0]
    tuned = Reconstruction(p, bp_nz=-1)
    nz, mb = tuned.autotune()  # cached: returns the choice made at create
    assert nz in (4, 8, 16) and mb in (2, 3, 4)
    ref = Reconstruction(p).run(fan)
    assert torch.equal(tuned.run(fan), ref)
