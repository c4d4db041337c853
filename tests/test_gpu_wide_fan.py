"""A wide-fan scan: the source is close enough (dso = 60 mm) that the volume's outer tiles see
|phat / dso| up to about 0.75, so the exact backprojector runs both of its column-angle forms in
one reconstruction -- the polynomial asin on tiles within dso / 2 of the axis and asinf on the
rest -- and both must match the FP64 oracle.  Bar: rel-L2 <= 1e-4 (FP32 volume)."""
import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu
from tests.test_gpu_pipeline import oracle_block_pipeline

pytestmark = pytest.mark.gpu


def test_wide_fan_exact_matches_fp64_oracle(cuda):
    import torch

    geo = ScanGeometry(ns=96, nt=8, ds=1.0, dt=1.0, npt=120, pitch=1.0, nx=64, ny=64, dx=1.0,
                       dz=1.0, dso=60.0).with_blocks(1)
    p = Plan(geo)
    corner = np.hypot(geo.nx / 2 * geo.dx, geo.ny / 2 * geo.dx)
    assert corner / geo.dso > 0.6  # outer tiles take asinf, central ones the polynomial
    z_lo, z_hi = p.blocks[0].block_start, p.blocks[-1].block_end
    ph = Phantom.random(5, seed=11, fov_radius=28.0, z_lo=z_lo, z_hi=z_hi, semi=(2.0, 10.0))
    fan = simulate_gpu(geo, ph, i0=1e5, seed=5).cpu().numpy()
    r = Reconstruction(p, mode=capi.MODE_BLOCK, interp=capi.INTERP_EXACT, addr=capi.ADDR_BORDER)
    img = r.run(torch.from_numpy(fan).cuda()).cpu().numpy()
    ref = oracle_block_pipeline(p, fan, orc.EXACT, orc.BORDER, orc.BORDER, 0)
    err = orc.rel_l2(img, ref)
    print(f"wide fan: rel_l2 vs FP64 oracle = {err:.3e}")
    assert np.isfinite(img).all()
    assert err < 1e-4
