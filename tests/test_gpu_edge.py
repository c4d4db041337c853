"""Edge cases on the GPU: a ragged geometry (odd column count, 7 detector rows, a 45 x 37 image,
slab widths that are no multiple of the tiles) through the whole pipeline in every filter mode
and from host and device buffers against the FP64 oracle, and empty inputs."""
import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ragged(cuda):
    geo = ScanGeometry(ns=97, nt=7, ds=1.0, dt=1.1, npt=130, pitch=0.9, nx=45, ny=37, dx=1.1,
                       dz=0.9).with_blocks(2)
    p = Plan(geo)
    zs = [b.block_start for b in p.blocks] + [b.block_end for b in p.blocks]
    ph = Phantom.random(6, seed=21, fov_radius=20.0, z_lo=min(zs), z_hi=max(zs), semi=(2.0, 9.0))
    fan = simulate_gpu(geo, ph, i0=1e5, seed=22)
    return p, fan


def _oracle(p, fan):
    g, ig = p.info.ctg, p.info.ig
    h = orc.ramp_taps(g.ns, g.ds)
    out = []
    for bi in p.blocks[: p.info.n_blocks_run]:
        blk = fan[bi.block_proj_start: bi.block_proj_start + g.n_angle_add]
        par = orc.rebin_fan2par(g, blk, orc.EXACT, orc.BORDER).astype(np.float32)
        f = orc.filter_rows(h, par.reshape(-1, g.ns), mode=0).reshape(par.shape).astype(np.float32)
        betas = p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        out.append(orc.bp_par(g, ig, betas, f, orc.EXACT, orc.BORDER))
    return np.concatenate(out, 0)


@pytest.mark.parametrize("fmode", [capi.FILTER_FP32, capi.FILTER_BF16X6])
@pytest.mark.parametrize("mode", [capi.MODE_SCAN, capi.MODE_BLOCK])
def test_ragged_geometry_matches_fp64_oracle(ragged, fmode, mode):
    import torch

    p, fan = ragged
    ref = _oracle(p, fan.cpu().numpy())
    rec = Reconstruction(p, mode=mode, interp=capi.INTERP_EXACT, filter_mode=fmode)
    img = rec.run(fan).cpu().numpy()
    err = orc.rel_l2(img, ref)
    print(f"ragged mode={mode} filter={fmode}: rel_l2 {err:.2e}")
    assert err < 1e-4  # the FP32-volume bar
    host = torch.empty(rec.image_shape, dtype=torch.float32).pin_memory()
    rec.run(fan.cpu().pin_memory(), host)
    assert np.array_equal(host.numpy(), img)


def test_empty_inputs(cuda):
    import torch

    lib = capi.load()
    h = torch.zeros(2 * 33, device="cuda")
    rows = torch.zeros(33, device="cuda")
    # zero rows: nothing to filter, in every mode
    for m in (capi.FILTER_FP32, capi.FILTER_BF16X3, capi.FILTER_BF16X6):
        assert lib.lct_filter_rows(33, h.data_ptr(), rows.data_ptr(), 0, m, None) == capi.LCT_OK
    # an empty view range simulates nothing
    ell = torch.zeros(16, dtype=torch.float64, device="cuda")
    ang = torch.zeros(4, dtype=torch.float64, device="cuda")
    fan = torch.zeros(4 * 2 * 8, device="cuda")
    assert lib.lct_sim_project(ell.data_ptr(), 1, 8, 2, 1.0, 1.0, 3.5, 0.5, 570.0, ang.data_ptr(),
                               ang.data_ptr(), 2, 2, 1e5, 1, fan.data_ptr(), None) == capi.LCT_OK
    torch.cuda.synchronize()
    assert lib.lct_device_status(None) in (capi.LCT_OK, capi.LCT_ERR_ARG)


def test_pi_original_chain_matches_fp64_oracle(ragged):
    """The PI-original path end to end (block mode: PI-original rebin, its pre-weighting, the
    FP32 filter, PI-window backprojection) on the ragged geometry against the oracle's chain."""
    p, fan = ragged
    g, ig = p.info.ctg, p.info.ig
    f = fan.cpu().numpy()
    h = orc.ramp_taps(g.ns, g.ds)
    ref = []
    for bi in p.blocks[: p.info.n_blocks_run]:
        blk = f[bi.block_proj_start: bi.block_proj_start + g.n_angle_add]
        par = orc.rebin_pi_ori(g, blk, orc.EXACT, orc.BORDER).astype(np.float32)
        par = orc.weight_pi_ori(g, par).astype(np.float32)
        flt = orc.filter_rows(h, par.reshape(-1, g.ns), mode=0).reshape(par.shape).astype(np.float32)
        betas = p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        ref.append(orc.bp_pi_ori(g, ig, betas, flt, orc.EXACT, orc.BORDER))
    ref = np.concatenate(ref, 0)
    rec = Reconstruction(p, mode=capi.MODE_BLOCK, interp=capi.INTERP_EXACT,
                         rebinner=capi.REBIN_PI_ORI, preweight=capi.PW_PI_ORI,
                         backprojector=capi.BP_PI_ORI)
    img = rec.run(fan).cpu().numpy()
    err = orc.rel_l2(img, ref)
    print(f"PI-original chain: rel_l2 {err:.2e}")
    assert err < 1e-4


@pytest.mark.parametrize("addr", [capi.ADDR_BORDER, capi.ADDR_LEGACY])
def test_pi_original_tex8_recon_matches_the_stage_chain(ragged, addr):
    """Block-mode PI-original chain in TEX8: lct_recon keeps one texture of the fan block for all
    its blocks (both addressings on one array; legacy addressing clamps the first block), the
    stage entry point lct_rebin_pi_ori binds a texture per call as the reference does.  Same
    kernels, same texels: the volumes are bit-identical."""
    import ctypes as C

    import torch

    p, fan = ragged
    g, ig = p.info.ctg, p.info.ig
    lib = capi.load()
    rec = Reconstruction(p, mode=capi.MODE_BLOCK, interp=capi.INTERP_TEX8, addr=addr,
                         rebinner=capi.REBIN_PI_ORI, preweight=capi.PW_PI_ORI,
                         backprojector=capi.BP_PI_ORI, filter_mode=capi.FILTER_FP32)
    img = rec.run(fan).cpu().numpy()
    taps = np.zeros(2 * g.ns, dtype=np.float32)  # the recon's own taps (lct_recon_opts defaults)
    capi.check(lib.lct_filter_taps(capi.FILTER_RAMLAK, capi.WINDOW_NONE, g.ns, g.ds,
                                   taps.ctypes.data))
    h = torch.from_numpy(taps).cuda()
    slab = 32 * ig.ny * ig.nx
    ref = np.empty(p.info.n_blocks_run * slab, dtype=np.float32)
    par = torch.empty(g.n_angle * g.nt * g.ns, dtype=torch.float32, device="cuda")
    out = torch.empty(slab, dtype=torch.float32, device="cuda")
    for b, bi in enumerate(p.blocks[: p.info.n_blocks_run]):
        a = capi.ADDR_CLAMP if (addr == capi.ADDR_LEGACY and b == 0) else capi.ADDR_BORDER
        blk = fan[bi.block_proj_start: bi.block_proj_start + g.n_angle_add].contiguous()
        betas = torch.from_numpy(np.ascontiguousarray(
            p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle])).cuda()
        capi.check(lib.lct_rebin_pi_ori(C.byref(g), blk.data_ptr(), par.data_ptr(),
                                        capi.INTERP_TEX8, a, None))
        capi.check(lib.lct_weight_pi_ori(C.byref(g), par.data_ptr(), None))
        capi.check(lib.lct_filter_rows(g.ns, h.data_ptr(), par.data_ptr(), g.n_angle * g.nt,
                                       capi.FILTER_FP32, None))
        capi.check(lib.lct_backproject_pi_ori(C.byref(g), C.byref(ig), betas.data_ptr(),
                                              par.data_ptr(), out.data_ptr(), capi.INTERP_TEX8,
                                              a, None))
        torch.cuda.synchronize()
        ref[b * slab:(b + 1) * slab] = out.cpu().numpy()
    assert np.isfinite(img).all()
    np.testing.assert_array_equal(img.ravel(), ref)
