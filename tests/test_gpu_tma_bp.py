"""The TMA-staged backprojector (each view's tile footprint of quads loaded into shared memory
by cp.async.bulk.tensor, samples read from there; warps whose samples leave the box read global
memory) against the quad kernel that samples through L1: the same arithmetic on the same quad
values, so the volumes must be bit-identical -- device-resident whole launches, streamed runs
(the first slab's parts stay on the L1 kernel) and bounded rings (box coordinates are ring
slots), on a toy scan and on config 1's detector (672 x 16, 256 x 256)."""
import numpy as np
import pytest

from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu

pytestmark = pytest.mark.gpu


def _scan(geo, nblocks, seed):
    g = geo.with_blocks(nblocks)
    p = Plan(g)
    lo = min(p.blocks[0].block_start, p.blocks[-1].block_end)
    hi = max(p.blocks[0].block_start, p.blocks[-1].block_end)
    fov = 0.5 * g.nx * g.dx
    ph = Phantom.random(8, seed=seed, fov_radius=fov, z_lo=lo, z_hi=hi,
                        semi=(0.1 * fov, 0.5 * fov))
    return p, simulate_gpu(g, ph, i0=1e5, seed=seed)


@pytest.mark.parametrize("which", ["toy", "config1"])
def test_tma_staged_backprojection_is_bit_identical(small_geo, cuda, which):
    import torch

    if which == "toy":
        p, fan = _scan(small_geo, 4, 41)
    else:
        geo = ScanGeometry(ns=672, nt=16, ds=1.0, dt=1.0, npt=1160, pitch=1.0, nx=256, ny=256,
                           dx=1.0, dz=1.0)
        p, fan = _scan(geo, 2, 42)
    kw = dict(mode=capi.MODE_SCAN, interp=capi.INTERP_EXACT, filter_mode=capi.FILTER_BF16X6,
              addr=capi.ADDR_BORDER)
    ref = Reconstruction(p, bp_sampler=capi.BP_SAMPLER_QUADS, **kw).run(fan)
    tma = Reconstruction(p, bp_sampler=capi.BP_SAMPLER_QUADS_TMA, **kw)
    assert torch.equal(tma.run(fan), ref)
    h_fan = fan.cpu().pin_memory()
    h_img = torch.full(tma.image_shape, float("nan"), dtype=torch.float32).pin_memory()
    tma.run(h_fan, h_img)  # streamed
    assert np.array_equal(h_img.numpy(), ref.cpu().numpy())
    b = Reconstruction(p, bounded=True, piece_views=32, bp_sampler=capi.BP_SAMPLER_QUADS_TMA, **kw)
    h_img.fill_(float("nan"))
    b.run(h_fan, h_img)
    assert np.array_equal(h_img.numpy(), ref.cpu().numpy())
    import ctypes as C

    code = C.c_int(0)
    capi.check(capi.load().lct_device_status(C.byref(code)))
    assert code.value == 0  # no bounded wait ran out
