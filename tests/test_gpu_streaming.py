"""Scan-mode runs from host buffers overlap the uploads, the per-slab compute and the downloads;
every view is still uploaded, rebinned and filtered once by the same kernels, so the volume must
be bit-identical to the device-resident run -- checked across interpolation, addressing (LEGACY
runs its first slab clamped, unpacked) and filter modes, and with the learned correction fused
(each slab corrected once its neighbours are backprojected)."""
import numpy as np
import pytest
import torch

from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def four_slabs(cuda):
    # 4 blocks, ~2,000 global views: several 512-view pieces per slab window
    geo = ScanGeometry(ns=160, nt=16, ds=1.0, dt=1.0, npt=480, pitch=1.0, nx=48, ny=40, dx=1.5,
                       dz=1.0).with_blocks(4)
    p = Plan(geo)
    zs = [b.block_start for b in p.blocks] + [b.block_end for b in p.blocks]
    ph = Phantom.random(8, seed=11, fov_radius=30.0, z_lo=min(zs), z_hi=max(zs), semi=(3.0, 15.0))
    fan = simulate_gpu(geo, ph, i0=1e5, seed=12)
    return p, fan


@pytest.mark.parametrize("interp,addr,fmode", [
    (capi.INTERP_EXACT, capi.ADDR_BORDER, capi.FILTER_BF16X6),
    (capi.INTERP_TEX8, capi.ADDR_LEGACY, capi.FILTER_FP32),
    (capi.INTERP_EXACT, capi.ADDR_CLAMP, capi.FILTER_BF16X3),
])
def test_streamed_host_run_equals_device_run(four_slabs, interp, addr, fmode):
    p, fan = four_slabs
    rec = Reconstruction(p, mode=capi.MODE_SCAN, interp=interp, addr=addr, filter_mode=fmode)
    dev = rec.run(fan).cpu()
    h_fan = fan.cpu().pin_memory()
    h_img = torch.empty(rec.image_shape, dtype=torch.float32).pin_memory()
    for _ in range(2):  # twice: events, streams and buffers are reused between runs
        h_img.fill_(np.nan)
        rec.run(h_fan, h_img)
        torch.cuda.synchronize()
        assert torch.equal(h_img, dev)
    # device image, host fan: streamed uploads, no downloads
    d_img = torch.full(rec.image_shape, np.nan, dtype=torch.float32, device="cuda")
    rec.run(h_fan, d_img)
    assert torch.equal(d_img.cpu(), dev)


def test_streamed_learned_run_equals_device_run(four_slabs):
    from listctrecons_b200.learn import CNN

    p, fan = four_slabs
    rec = Reconstruction(p, mode=capi.MODE_SCAN, interp=capi.INTERP_EXACT,
                         filter_mode=capi.FILTER_BF16X6)
    net = CNN(16, p.info.ig.ny, p.info.ig.nx, train=False, seed=5)
    net.set_scales(0.5, 50.0)
    rec.set_learned(net, bound=0.05)
    dev = rec.run(fan).cpu()
    rej_dev = rec.learned_info()["rejected"]
    h_img = torch.full(rec.image_shape, np.nan, dtype=torch.float32).pin_memory()
    rec.run(fan.cpu().pin_memory(), h_img)
    assert torch.equal(h_img, dev)
    assert rec.learned_info()["rejected"] == rej_dev
