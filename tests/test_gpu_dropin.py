"""The drop-in reference program (reference host code + Stages.cpp + liblct.so) against the
reference program built from its own sources (oracle/_ref/ref_timed), same .prm and files.
Bar: images within rel-L2 1e-4; the filtered block (rebin.raw) within 1e-5 (TEX8 sampling and
the FP32 filter in the reference's order on both sides)."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DROPIN = ROOT / "listctrecons_b200" / "dropin" / "_build" / "LISTCTRecons"
REF = ROOT / "oracle" / "_ref" / "ref_timed"


@pytest.mark.skipif(not (DROPIN.exists() and REF.exists()), reason="builds need the reference tree")
@pytest.mark.parametrize("filt", ["fp32", "bf16x6"])
def test_dropin_matches_reference_program(cuda, tmp_path, filt):
    from listctrecons_b200.scan import write_scan_files
    from tests.golden.make_gpu_golden import small_scan

    geo, _, fan = small_scan()
    prm_ref = write_scan_files(geo, fan, tmp_path / "data", tmp_path / "ref")
    r = subprocess.run([str(REF), str(prm_ref)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-1500:]
    # the same scan, output to another directory, through the drop-in
    txt = prm_ref.read_text().replace(str(tmp_path / "ref"), str(tmp_path / "dropin"))
    (tmp_path / "dropin").mkdir()
    prm_d = tmp_path / "data" / "dropin.prm"
    prm_d.write_text(txt)
    env = dict(os.environ, LCT_DROPIN_FILTER=filt)
    d = subprocess.run([str(DROPIN), str(prm_d)], capture_output=True, text=True, timeout=600, env=env)
    assert d.returncode == 0, d.stdout[-1500:]
    assert "[ERROR]" not in d.stdout
    a = np.fromfile(tmp_path / "ref" / "image.raw", dtype=np.float32)
    b = np.fromfile(tmp_path / "dropin" / "image.raw", dtype=np.float32)
    ra = np.fromfile(tmp_path / "ref" / "rebin.raw", dtype=np.float32)
    rb = np.fromfile(tmp_path / "dropin" / "rebin.raw", dtype=np.float32)
    err, errf = orc.rel_l2(b, a), orc.rel_l2(rb, ra)
    print(f"drop-in ({filt}) vs reference program: image rel_l2={err:.3e}, filtered {errf:.3e}")
    assert a.size == b.size and err < 1e-4
    assert errf < 1e-5


TYPED = ROOT / "listctrecons_b200" / "dropin" / "_build" / "LISTCTRecons_b200"


def _typed_run(prm_src: Path, out_dir: Path, rtype: str, env_extra: dict) -> tuple[np.ndarray, dict]:
    """LISTCTRecons_b200 on a copy of prm_src writing to out_dir; (image, its JSON record)."""
    import json

    out_dir.mkdir()
    txt = prm_src.read_text()
    for line in txt.splitlines():
        if line.startswith("OutputDir:"):
            txt = txt.replace(line, f"OutputDir: {out_dir}/")
    prm = out_dir / "scan.prm"
    prm.write_text(txt)
    env = dict(os.environ, **env_extra)
    d = subprocess.run([str(TYPED), str(prm), rtype], capture_output=True, text=True, timeout=900,
                       env=env)
    assert d.returncode == 0, d.stdout[-1500:]
    assert "[ERROR]" not in d.stdout, d.stdout[-1500:]
    rec = json.loads(d.stdout.strip().splitlines()[-1])
    return np.fromfile(out_dir / "image.raw", dtype=np.float32), rec


@pytest.mark.skipif(not (TYPED.exists() and REF.exists()), reason="builds need the reference tree")
def test_factory_types_through_the_reference_interfaces(cuda, tmp_path):
    """The typed drop-in program builds its reconstructor with the reference's factory call
    (ReconstrctorAbstractFactory::createReconstructor) and runs Reconstructor::reconstruct:
      * "Helicalfdkramprebingpu" -- the drop-in stages, per block -- matches the reference
        program built from its own sources (rel-L2 < 1e-4);
      * "Helicalfdkramprebinb200" -- the whole-scan path, every view read once from the raw file
        with 64-bit offsets -- in the reference's sampling (TEX8, FP32 filter, its legacy
        first-block addressing) matches the reference program (rel-L2 < 1e-4), and in its default
        mode (exact, BF16x6, bounded memory) matches the FP64 oracle (rel-L2 < 1e-4)."""
    from listctrecons_b200.recon import Plan
    from listctrecons_b200.scan import write_scan_files
    from tests.golden.make_gpu_golden import small_scan

    geo, _, fan = small_scan()
    prm = write_scan_files(geo, fan, tmp_path / "data", tmp_path / "ref")
    r = subprocess.run([str(REF), str(prm)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-1500:]
    ref = np.fromfile(tmp_path / "ref" / "image.raw", dtype=np.float32)

    stages, rec = _typed_run(prm, tmp_path / "stages", "Helicalfdkramprebingpu",
                             {"LCT_DROPIN_FILTER": "fp32"})
    assert rec["type"] == "Helicalfdkramprebingpu"
    err = orc.rel_l2(stages, ref)
    print(f"typed program, reference type vs reference program: rel_l2={err:.3e}")
    assert stages.size == ref.size and err < 1e-4

    same, _ = _typed_run(prm, tmp_path / "b200_ref_sampling", "Helicalfdkramprebinb200",
                         {"LCT_DROPIN_INTERP": "tex8", "LCT_DROPIN_FILTER": "fp32",
                          "LCT_DROPIN_ADDR": "legacy"})
    err = orc.rel_l2(same, ref)
    print(f"whole-scan type (tex8, fp32, legacy) vs reference program: rel_l2={err:.3e}")
    assert same.size == ref.size and err < 1e-4

    fast, _ = _typed_run(prm, tmp_path / "b200", "Helicalfdkramprebinb200", {})
    p = Plan(geo)
    g, ig = p.info.ctg, p.info.ig
    h = orc.ramp_taps(g.ns, g.ds)
    vols = []
    for b in range(p.info.n_blocks):
        bi = p.blocks[b]
        blk = fan[bi.block_proj_start: bi.block_proj_start + g.n_angle_add]
        par = orc.rebin_fan2par(g, blk, orc.EXACT).astype(np.float32)
        f = orc.filter_rows_fp64(h, par).astype(np.float32)
        betas = p.angles32[bi.block_proj_start + g.add_projections:][: g.n_angle]
        vols.append(orc.bp_par_cols(g, ig, betas, f, orc.EXACT))
    oracle = np.concatenate(vols, 0).ravel()
    err = orc.rel_l2(fast, oracle)
    print(f"whole-scan type (exact, bf16x6, bounded) vs FP64 oracle: rel_l2={err:.3e}; "
          f"vs reference program {orc.rel_l2(fast, ref):.3e}")
    assert fast.size == oracle.size and err < 1e-4


@pytest.mark.skipif(not (TYPED.exists() and REF.exists()), reason="builds need the reference tree")
def test_pi_original_type_matches_the_references_pi_configuration(cuda, tmp_path):
    """The reference's alternate configuration (Src/ReconstructorAbstractFactory.cpp:19-22:
    PiOriRebiner, PiOriPreWeighting, RampFilterGPU, PiOriBackprojectorGPU), built from the
    reference's own classes and kernels (`ref_timed <prm> pi`), against the same configuration on
    the drop-in stages (`LISTCTRecons_b200 <prm> Helicalfdkpiorigpu`: the PI-original rebin sampled
    by the texture unit, the FP32 filter in the reference's order, the PI-window backprojector),
    same scan and files.  The reference's PI window has no bound against n_angle
    (CUDA/Backprojector.cu:225); on this scan a_middle + n_proj_turn / 2 stays below n_angle for
    every slice, so its view index never passes the end of its betas."""
    from listctrecons_b200.recon import Plan
    from listctrecons_b200.scan import write_scan_files
    from tests.golden.make_gpu_golden import small_scan

    geo, _, fan = small_scan()
    p = Plan(geo)
    g, ig = p.info.ctg, p.info.ig
    dzv = np.float32(g.pitch) / np.float32(g.n_proj_turn)
    for iz in range(ig.nz):  # the bound above, checked on the host before the reference runs
        zc = np.float32((iz - ig.wz) * ig.dz)
        a_mid = min(max(int(np.round((zc - np.float32(g.source_z0)) / dzv)), 0), g.n_angle - 1)
        assert a_mid + g.n_proj_turn // 2 <= g.n_angle - 1
    prm = write_scan_files(geo, fan, tmp_path / "data", tmp_path / "ref")
    r = subprocess.run([str(REF), str(prm), "pi"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-1500:]
    assert json_last(r.stdout)["chain"] == "pi_original"
    ref = np.fromfile(tmp_path / "ref" / "image.raw", dtype=np.float32)
    img, rec = _typed_run(prm, tmp_path / "pi", "Helicalfdkpiorigpu", {"LCT_DROPIN_FILTER": "fp32"})
    assert rec["type"] == "Helicalfdkpiorigpu"
    err = orc.rel_l2(img, ref)
    print(f"PI-original type vs the reference's PI configuration: rel_l2={err:.3e}, "
          f"max_abs={np.abs(img - ref).max():.3e}")
    assert img.size == ref.size and np.isfinite(ref).all() and err < 1e-4


def json_last(stdout: str) -> dict:
    import json

    return json.loads(stdout.strip().splitlines()[-1])
