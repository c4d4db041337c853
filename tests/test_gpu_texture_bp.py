"""The texture-unit backprojector (TEX8 through tex3D on a 3-D array of the filtered views, the
reference's own fetch) against the quad backprojector that emulates the unit's 8-bit weights in
registers, and both against the oracle's texture emulation.  The emulation rule is pinned to the
hardware (tests/test_gpu_texture.py), so the two samplers agree far below the 1e-4 bar; a bounded
(ring) texture run is bit-identical to the whole-scan texture run."""
import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, simulate_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scan(small_geo, cuda):
    geo = small_geo.with_blocks(5)
    p = Plan(geo)
    lo = min(p.blocks[0].block_start, p.blocks[-1].block_end)
    hi = max(p.blocks[0].block_start, p.blocks[-1].block_end)
    ph = Phantom.random(6, seed=33, fov_radius=14.0, z_lo=lo, z_hi=hi, semi=(2.0, 9.0))
    fan = simulate_gpu(geo, ph, i0=1e5, seed=8)
    return dict(plan=p, fan=fan)


def _oracle(p, fan):
    g, ig = p.info.ctg, p.info.ig
    h = orc.ramp_taps(g.ns, g.ds)
    out = []
    for b in range(p.info.n_blocks_run):
        bi = p.blocks[b]
        blk = fan[bi.block_proj_start: bi.block_proj_start + g.n_angle_add]
        par = orc.rebin_fan2par(g, blk, orc.TEXEMU).astype(np.float32)
        f = orc.filter_rows(h, par.reshape(-1, g.ns), mode=1).reshape(par.shape).astype(np.float32)
        betas = p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        out.append(orc.bp_par_cols(g, ig, betas, f, orc.TEXEMU))
    return np.concatenate(out, 0)


@pytest.mark.parametrize("mode", [capi.MODE_BLOCK, capi.MODE_SCAN])
def test_texture_sampler_matches_quads_and_oracle(scan, mode):
    p, fan = scan["plan"], scan["fan"]
    kw = dict(mode=mode, interp=capi.INTERP_TEX8, filter_mode=capi.FILTER_FP32,
              addr=capi.ADDR_BORDER)
    tex = Reconstruction(p, bp_sampler=capi.BP_SAMPLER_TEXTURE, **kw).run(fan).cpu().numpy()
    quad = Reconstruction(p, bp_sampler=capi.BP_SAMPLER_QUADS, **kw).run(fan).cpu().numpy()
    ref = _oracle(p, fan.cpu().numpy()) if mode == capi.MODE_BLOCK else None
    d = orc.rel_l2(tex, quad)
    print(f"mode={mode}: texture vs quads rel_l2={d:.3e}")
    assert d < 1e-5
    if ref is not None:
        e = orc.rel_l2(tex, ref)
        print(f"texture vs oracle (texture emulation): rel_l2={e:.3e}")
        assert e < 1e-4


def test_texture_sampler_streamed_and_bounded_are_bit_identical(scan):
    import torch

    p, fan = scan["plan"], scan["fan"]
    kw = dict(mode=capi.MODE_SCAN, interp=capi.INTERP_TEX8, filter_mode=capi.FILTER_BF16X6,
              addr=capi.ADDR_CLAMP, bp_sampler=capi.BP_SAMPLER_TEXTURE)
    ref = Reconstruction(p, **kw).run(fan).cpu().numpy()
    h_fan = fan.cpu().pin_memory()
    h_img = torch.empty(ref.shape, dtype=torch.float32).pin_memory()
    Reconstruction(p, **kw).run(h_fan, h_img)  # streamed host run (texture filled per piece)
    np.testing.assert_array_equal(h_img.numpy(), ref)
    b = Reconstruction(p, bounded=True, piece_views=24, **kw)
    h_img.fill_(float("nan"))
    b.run(h_fan, h_img)
    np.testing.assert_array_equal(h_img.numpy(), ref)
