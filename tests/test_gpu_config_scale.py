"""Parity at the benchmark configurations' real geometries (not toy scans).

  * config 1 -- 672 x 16 detector at 1 mm, 1160 views/rotation, pitch 1, 256 x 256 x 32 at 1 mm,
    the shortest scan the reference planner gives 32 slices (3.70 rotations):
      - scan mode, exact interpolation, BF16x6 tensor-core filter against the FP64 oracle;
      - block mode, TEX8 sampling, FP32 filter against the oracle's texture emulation;
      - the drop-in program (reference host code + the product's stages) against the reference
        program built from its own sources, on the same files;
  * config 3 -- one scan of each row count {16, 32, 64} with config 3's column counts, pitches
    and views per rotation, reconstructed together through the batched path (one graph launch
    per stage), each against the FP64 oracle.

The oracle rebins each block's own fan window, filters in FP64 and backprojects every voxel
(tests/test_oracle_kat.py pins its column-order backprojector to the voxel-order one bit for bit).
Bar: rel-L2 <= 1e-4 for FP32 volumes, written in each assert."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi
from listctrecons_b200.recon import Batch, Plan, Reconstruction
from listctrecons_b200.scan import Phantom, ScanGeometry, simulate_gpu, write_scan_files

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DROPIN = ROOT / "listctrecons_b200" / "dropin" / "_build" / "LISTCTRecons"
REF = ROOT / "oracle" / "_ref" / "ref_timed"

CFG1 = dict(ns=672, nt=16, ds=1.0, dt=1.0, npt=1160, pitch=1.0, nx=256, ny=256, dx=1.0, dz=1.0)


def oracle_volume(plan, fan, f0, interp, kind=capi.FILTER_RAMLAK, addr=orc.BORDER):
    """FP64 oracle of every block the plan runs: rebin the block's fan window, FP64 filter,
    column-order backprojection.  fan holds views from f0 on (host array)."""
    g, ig = plan.info.ctg, plan.info.ig
    h = orc.shepp_logan_taps(g.ns, g.ds) if kind == capi.FILTER_SHEPP_LOGAN else orc.ramp_taps(g.ns, g.ds)
    out = []
    for b in range(plan.info.first_block, plan.info.first_block + plan.info.n_blocks_run):
        bi = plan.blocks[b]
        blk = fan[bi.block_proj_start - f0: bi.block_proj_start - f0 + g.n_angle_add]
        par = orc.rebin_fan2par(g, blk, interp, addr).astype(np.float32)
        f = orc.filter_rows_fp64(h, par).astype(np.float32)
        betas = plan.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        out.append(orc.bp_par_cols(g, ig, betas, f, interp, addr))
    return np.concatenate(out, 0)


@pytest.fixture(scope="module")
def cfg1(cuda):
    geo = ScanGeometry(**CFG1).with_blocks(1, cap=False)
    plan = Plan(geo)
    assert plan.info.n_blocks == 1 and geo.readings == 4290  # 3.70 rotations plan 32 slices
    bi = plan.blocks[0]
    lo, hi = sorted((bi.block_start, bi.block_end))
    ph = Phantom.head_like(seed=11, fov_radius=0.5 * CFG1["nx"] * CFG1["dx"], z_lo=lo, z_hi=hi)
    fan = simulate_gpu(geo, ph, i0=1e5, seed=5)
    return dict(geo=geo, plan=plan, fan=fan, fan_np=fan.cpu().numpy())


def test_cfg1_scan_exact_bf16x6_matches_fp64_oracle(cfg1):
    p = cfg1["plan"]
    r = Reconstruction(p, mode=capi.MODE_SCAN, interp=capi.INTERP_EXACT,
                       filter_mode=capi.FILTER_BF16X6)
    img = r.run(cfg1["fan"]).cpu().numpy()
    ref = oracle_volume(p, cfg1["fan_np"], 0, orc.EXACT)
    err = orc.rel_l2(img, ref)
    print(f"config 1, scan/exact/bf16x6 vs FP64 oracle: rel_l2={err:.3e} max_abs={orc.max_abs(img, ref):.3e}")
    assert err < 1e-4


def test_cfg1_block_tex8_fp32_matches_texture_oracle(cfg1):
    p = cfg1["plan"]
    r = Reconstruction(p, mode=capi.MODE_BLOCK, interp=capi.INTERP_TEX8,
                       filter_mode=capi.FILTER_FP32)
    img = r.run(cfg1["fan"]).cpu().numpy()
    ref = oracle_volume(p, cfg1["fan_np"], 0, orc.TEXEMU)
    err = orc.rel_l2(img, ref)
    print(f"config 1, block/tex8/fp32 vs oracle (texture emulation): rel_l2={err:.3e}")
    assert err < 1e-4


@pytest.mark.skipif(not (DROPIN.exists() and REF.exists()), reason="builds need the reference tree")
def test_cfg1_dropin_matches_reference_program(cfg1, tmp_path):
    prm_ref = write_scan_files(cfg1["geo"], cfg1["fan_np"], tmp_path / "data", tmp_path / "ref")
    r = subprocess.run([str(REF), str(prm_ref)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-1500:]
    txt = prm_ref.read_text().replace(str(tmp_path / "ref"), str(tmp_path / "dropin"))
    (tmp_path / "dropin").mkdir()
    prm_d = tmp_path / "data" / "dropin.prm"
    prm_d.write_text(txt)
    env = dict(os.environ, LCT_DROPIN_FILTER="fp32")
    d = subprocess.run([str(DROPIN), str(prm_d)], capture_output=True, text=True, timeout=900, env=env)
    assert d.returncode == 0, d.stdout[-1500:]
    assert "[ERROR]" not in d.stdout
    a = np.fromfile(tmp_path / "ref" / "image.raw", dtype=np.float32)
    b = np.fromfile(tmp_path / "dropin" / "image.raw", dtype=np.float32)
    ra = np.fromfile(tmp_path / "ref" / "rebin.raw", dtype=np.float32)
    rb = np.fromfile(tmp_path / "dropin" / "rebin.raw", dtype=np.float32)
    err, errf = orc.rel_l2(b, a), orc.rel_l2(rb, ra)
    print(f"config 1, drop-in vs reference program: image rel_l2={err:.3e}, filtered {errf:.3e}")
    assert a.size == b.size == 32 * 256 * 256
    assert err < 1e-4
    assert errf < 1e-5


# config 3 shapes: rows {16, 32, 64}, 672-896 columns, pitch in [0.5, 1.5], 1000-1200 views/rot
CFG3 = [
    dict(ns=672, nt=16, ds=0.6, dt=0.6, npt=1000, pitch=0.5, nx=256, ny=256, dx=1.0, dz=0.5),
    dict(ns=800, nt=32, ds=0.5, dt=0.5, npt=1200, pitch=1.0, nx=256, ny=256, dx=1.0, dz=0.75),
    dict(ns=896, nt=64, ds=0.5, dt=0.5, npt=1152, pitch=1.5, nx=256, ny=256, dx=1.0, dz=1.0),
]


def test_cfg3_batch_each_row_count_matches_fp64_oracle(cuda):
    import torch

    plans, fans, phs = [], [], []
    for i, c in enumerate(CFG3):
        geo = ScanGeometry(**c).with_blocks(1)
        p = Plan(geo)
        bi = p.blocks[0]
        lo, hi = sorted((bi.block_start, bi.block_end))
        ph = Phantom.random(10, seed=500 + i, fov_radius=0.5 * c["nx"] * c["dx"], z_lo=lo, z_hi=hi,
                            semi=(5.0, 60.0))
        plans.append(p)
        fans.append((geo, ph))
    b = Batch(plans, interp=capi.INTERP_EXACT, filter_mode=capi.FILTER_BF16X6)
    dev_fans, v0 = [], []
    for (geo, ph), (f0, fc) in zip(fans, b.fan_ranges):
        dev_fans.append(simulate_gpu(geo, ph, i0=1e5, seed=7, v0=f0, v1=f0 + fc))
        v0.append(f0)
    imgs = b.run(dev_fans, fan_view0=v0)
    torch.cuda.synchronize()
    for p, img, f, f0 in zip(plans, imgs, dev_fans, v0):
        ref = oracle_volume(p, f.cpu().numpy(), f0, orc.EXACT)
        got = img.cpu().numpy()
        err = orc.rel_l2(got, ref)
        print(f"config 3 scan nt={p.info.ctg.nt} ns={p.info.ctg.ns}: rel_l2={err:.3e}")
        assert err < 1e-4
