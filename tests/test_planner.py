"""Planner parity: the product's restatement of ReconData::convert_from_file_params and
BlockInfo::update against the reference's own compiled code (tests/golden/plans.json, made by
tests/golden/make_golden.py from oracle/_ref/ref_plan)."""
import ctypes as C
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan

GOLD = Path(__file__).resolve().parent / "golden"
from tests.golden.make_golden import CASES, case_arrays, case_prm_values, write_case  # noqa: E402

PLANS = json.loads((GOLD / "plans.json").read_text())


def _params(c):
    v = case_prm_values(c)
    p = capi.ScanParams()
    p.ns, p.nt, p.ds, p.dt, p.pitch_value = v["Ns"], v["Nt"], v["Ds"], v["Dt"], v["PitchValue"]
    p.nx, p.ny, p.dx, p.dz = v["Nx"], v["Ny"], v["Dx"], v["Dz"]
    p.offset_x, p.offset_y = v["OffsetX"], v["OffsetY"]
    p.readings, p.view_offset, p.data_offset = v["Readings"], 0, 0
    p.r_src_to_iso, p.central_channel, p.n_proj_turn = v["RSrcToIso"], v["CentralChannel"], v["NProjTurn"]
    return p


def _plan(c):
    ang, z, _ = case_arrays(c)
    return Plan(params=_params(c), angles32=ang, zpos32=z)


def _f(x):
    return float(np.float32(x))


@pytest.mark.parametrize("rec", PLANS, ids=[r["case"]["name"] for r in PLANS])
def test_planner_matches_reference(rec):
    c = rec["case"]
    if "error" in rec:
        if "outside of allowed data range" in rec["error"]:
            with pytest.raises(capi.LctError) as e:
                _plan(c)
            assert e.value.status == capi.LCT_ERR_RANGE
        else:
            # the reference aborts sizing its image in int (cfg5); the product plans it in 64 bit
            p = _plan(c)
            assert p.info.n_blocks == 93 and p.info.n_slices_recon == 2976
            assert p.info.ig.nx * p.info.ig.ny * p.info.n_slices_recon > 2**31
        return
    ref = rec["ref"]
    p = _plan(c)
    g = p.info.ctg
    for k, v in ref["ctg"].items():
        got = getattr(g, k)
        assert (got == v) if isinstance(v, int) else (_f(got) == _f(v)), (k, got, v)
    for k, v in ref["ig"].items():
        got = getattr(p.info.ig, k)
        assert (got == v) if isinstance(v, int) else (_f(got) == _f(v)), (k, got, v)
    for k, v in ref["ri"].items():
        got = getattr(p.info, k)
        assert (got == v) if isinstance(v, int) else (_f(got) == _f(v)), (k, got, v)
    assert p.info.n_blocks == len(ref["blocks"]) == len(p.blocks)
    for b, rb in zip(p.blocks, ref["blocks"]):
        assert b.block_idx == rb["block_idx"]
        assert b.block_proj_start == rb["block_proj_start"]
        assert b.block_proj_end == rb["block_proj_end"]
        assert _f(b.block_start) == _f(rb["block_start"])
        assert _f(b.block_end) == _f(rb["block_end"])
        assert b.block_slice_start == rb["block_slice_start"]
        assert b.block_slice_end == rb["block_slice_end"]


def test_cfg5_windows_match_reference_small_image():
    big = [r for r in PLANS if r["case"]["name"] == "cfg5_20rot"][0]
    small = [r for r in PLANS if r["case"]["name"] == "cfg5_20rot_img256"][0]["ref"]
    p = _plan(big["case"])
    assert [b.block_proj_start for b in p.blocks] == [b["block_proj_start"] for b in small["blocks"]]
    assert p.info.ctg.n_angle == small["ctg"]["n_angle"]


def test_max_blocks_caps_run_only():
    c = [r for r in PLANS if r["case"]["name"] == "cfg2_10rot"][0]["case"]
    ang, z, _ = case_arrays(c)
    prm = _params(c)
    prm.max_blocks = 8
    p = Plan(params=prm, angles32=ang, zpos32=z)
    assert p.info.n_blocks == 16 and p.info.n_blocks_run == 8


def test_planner_rejects_bad_input():
    c = [r for r in PLANS if r["case"]["name"] == "small_test"][0]["case"]
    ang, z, _ = case_arrays(c)
    prm = _params(c)
    prm.readings = 50
    with pytest.raises(capi.LctError):
        Plan(params=prm, angles32=ang, zpos32=z)
    flat = np.zeros_like(z)
    with pytest.raises(capi.LctError):
        Plan(params=_params(c), angles32=ang, zpos32=flat)


REF_PLAN = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "ref_plan"


@pytest.mark.skipif(not REF_PLAN.exists(), reason="reference build (oracle/_ref) not present")
def test_random_geometries_against_reference_binary():
    rng = np.random.default_rng(7)
    for _ in range(12):
        c = dict(name="rand", ns=int(rng.integers(64, 900)), nt=int(rng.choice([8, 16, 32, 64])),
                 ds=float(rng.uniform(0.4, 1.2)), dt=float(rng.uniform(0.4, 1.2)),
                 npt=int(rng.integers(100, 1500)), pitch=float(rng.uniform(0.5, 1.5)),
                 rot=float(rng.uniform(4, 9)), nx=64, ny=64, dx=float(rng.uniform(0.3, 1.5)),
                 dz=float(rng.uniform(0.3, 1.5)), z_dir=int(rng.choice([1, -1])),
                 z_start=float(rng.uniform(-300, 300)), start=float(rng.uniform(0, 6.28)))
        with tempfile.TemporaryDirectory() as td:
            prm = write_case(c, Path(td))
            r = subprocess.run([str(REF_PLAN), "plan", str(prm)], capture_output=True, text=True)
        if r.returncode != 0:
            with pytest.raises(capi.LctError):
                _plan(c)
            continue
        ref = json.loads(r.stdout[r.stdout.index("{\"ctg\""):])
        p = _plan(c)
        assert [b.block_proj_start for b in p.blocks] == [b["block_proj_start"] for b in ref["blocks"]]
        assert p.info.ctg.n_angle == ref["ctg"]["n_angle"]
        assert p.info.ctg.add_projections == ref["ctg"]["add_projections"]
        assert _f(p.info.recon_start_pos) == _f(ref["ri"]["recon_start_pos"])


def test_adopted_plan_runs_the_given_blocks():
    """lct_plan_adopt keeps exactly the planner results it is given (the drop-in whole-scan
    reconstructor adopts the reference planner's ReconData and BlockInfos this way)."""
    import ctypes as C

    from listctrecons_b200 import capi
    from listctrecons_b200.recon import Plan
    from listctrecons_b200.scan import ScanGeometry

    geo = ScanGeometry(ns=736, nt=64, ds=0.6, dt=0.6, npt=1152, pitch=0.8, nx=512, ny=512,
                       dx=0.5, dz=0.5, readings=11520)
    p = Plan(geo)
    lib = capi.load()
    info = capi.PlanInfo()
    C.memmove(C.byref(info), C.byref(p.info), C.sizeof(info))
    info.first_block, info.n_blocks_run = 3, 5
    blocks = (capi.BlockInfo * len(p.blocks))(*p.blocks)
    h = C.c_void_p()
    capi.check(lib.lct_plan_adopt(C.byref(info), blocks, len(p.blocks), p.angles32.ctypes.data,
                                  p.zpos32.ctypes.data, C.byref(h)))
    got = capi.PlanInfo()
    capi.check(lib.lct_plan_info_get(h, C.byref(got)))
    assert bytes(got) == bytes(info)
    for b in range(len(p.blocks)):
        bi = capi.BlockInfo()
        capi.check(lib.lct_plan_block(h, b, C.byref(bi)))
        assert bytes(bi) == bytes(p.blocks[b])
    lib.lct_plan_destroy(h)
    # inconsistent inputs are refused
    bad = capi.PlanInfo()
    C.memmove(C.byref(bad), C.byref(info), C.sizeof(bad))
    bad.n_blocks_run = len(p.blocks)  # first_block 3 + all blocks runs past the end
    assert lib.lct_plan_adopt(C.byref(bad), blocks, len(p.blocks), p.angles32.ctypes.data,
                              p.zpos32.ctypes.data, C.byref(h)) == capi.LCT_ERR_ARG
    assert lib.lct_plan_adopt(C.byref(info), blocks, len(p.blocks) - 1, p.angles32.ctypes.data,
                              p.zpos32.ctypes.data, C.byref(h)) == capi.LCT_ERR_ARG
