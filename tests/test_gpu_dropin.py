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
