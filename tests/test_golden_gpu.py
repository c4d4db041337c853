"""The oracle against outputs recorded on a B200 (tests/golden/make_gpu_golden.py):
the texture unit's linear filter, and the reference's own CUDA path on a small scan."""
from pathlib import Path

import numpy as np
import pytest

import oracle as orc

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.skipif(not (GOLD / "tex_hw.npz").exists(), reason="fixture not generated yet")
def test_oracle_texture_emulation_matches_hardware():
    d = np.load(GOLD / "tex_hw.npz")
    x = d["ramp_x"]
    ramp = np.tile(np.arange(64, dtype=np.float32), (2, 2, 1))
    c1 = np.stack([x, np.full_like(x, 0.5), np.full_like(x, 0.5)], 1)
    assert np.abs(orc.tex3d_sample(ramp, c1, orc.TEXEMU) - d["ramp_hw"]).max() < 1e-5
    emu = orc.tex3d_sample(d["bil_vol"], d["bil_coord"], orc.TEXEMU, orc.BORDER)
    assert np.abs(emu - d["bil_hw"]).max() < 1e-6
    exact = orc.tex3d_sample(d["bil_vol"], d["bil_coord"], orc.EXACT, orc.BORDER)
    assert np.abs(exact - d["bil_hw"]).max() > 1e-3  # the rule matters


@pytest.mark.skipif(not (GOLD / "ref_gpu_small.npz").exists(), reason="fixture not generated yet")
def test_oracle_pipeline_matches_reference_cuda_path():
    from tests.golden.make_gpu_golden import small_scan
    from listctrecons_b200.recon import Plan

    d = np.load(GOLD / "ref_gpu_small.npz")
    geo, _, fan = small_scan()
    p = Plan(geo)
    g, ig = p.info.ctg, p.info.ig
    h = orc.ramp_taps(g.ns, g.ds)
    out = []
    for b, bi in enumerate(p.blocks):
        addr = orc.CLAMP if b == 0 else orc.BORDER  # legacy binding: clamp until the 2nd bind
        blk = fan[bi.block_proj_start: bi.block_proj_start + g.n_angle_add]
        par = orc.rebin_fan2par(g, blk, orc.TEXEMU, addr).astype(np.float32)
        f = orc.filter_rows(h, par.reshape(-1, g.ns), mode=1).reshape(par.shape).astype(np.float32)
        if b == len(p.blocks) - 1:
            head = f.reshape(-1)[: d["rebin_head"].size]
            assert orc.rel_l2(head, d["rebin_head"]) < 1e-6
        betas = p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        out.append(orc.bp_par(g, ig, betas, f, orc.TEXEMU, addr))
    img = np.concatenate(out).reshape(-1)
    err = orc.rel_l2(img, d["image"])
    print(f"oracle vs reference CUDA path: rel_l2={err:.3e}")
    assert err < 1e-4
