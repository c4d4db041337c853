"""Generates tests/golden/{plans,taps}.json from the reference's own host code.

Runs oracle/_ref/ref_plan -- the reference's Src/DataStructs.cpp, Src/FileParams.cpp and
Src/Filter.cpp compiled from the reference tree by `make -C oracle ref` -- on scans written in
the reference's file formats, and records what it prints: the CTGeom / ImgGeom / ReconInfo of
ReconData(fp) and every block's BlockInfo, or the fact that it exits with an error.  The angle
and couch files are regenerated by the tests from the recorded case parameters (see
`case_arrays`), so the fixtures stay small.

    python tests/golden/make_golden.py        (needs the reference tree; run in the build
                                               container, the outputs are committed)
"""
from __future__ import annotations

import json
import math
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF_PLAN = ROOT / "oracle" / "_ref" / "ref_plan"

# (name, geometry) -- shapes of the benchmark configurations plus edge cases
CASES = [
    # small helical scan, 672x16 @1.0, 1160 views/rot, pitch 1, 256^2 @1 mm
    dict(name="cfg1_3rot", ns=672, nt=16, ds=1.0, dt=1.0, npt=1160, pitch=1.0, rot=3.0, nx=256, ny=256, dx=1.0, dz=1.0),
    dict(name="cfg1_ext", ns=672, nt=16, ds=1.0, dt=1.0, npt=1160, pitch=1.0, views=4290, nx=256, ny=256, dx=1.0, dz=1.0),
    # split-precision config, 736x64 @0.6, 1152 views/rot, pitch 0.8, 10 rot, 512^2 @0.5
    dict(name="cfg2_10rot", ns=736, nt=64, ds=0.6, dt=0.6, npt=1152, pitch=0.8, rot=10.0, nx=512, ny=512, dx=0.5, dz=0.5),
    dict(name="cfg4_4rot", ns=736, nt=64, ds=0.6, dt=0.6, npt=1152, pitch=1.5, rot=4.0, nx=256, ny=256, dx=1.0, dz=1.0),
    # the reference itself overflows int sizing the 1024^2 x 2976-slice image
    # (Src/DataStructs.cpp:246) and aborts; the same scan with a 256^2 image pins its windows
    dict(name="cfg5_20rot", ns=896, nt=128, ds=0.5, dt=0.5, npt=2304, pitch=1.0, rot=20.0, nx=1024, ny=1024, dx=0.4, dz=0.4),
    dict(name="cfg5_20rot_img256", ns=896, nt=128, ds=0.5, dt=0.5, npt=2304, pitch=1.0, rot=20.0, nx=256, ny=256, dx=0.4, dz=0.4),
    dict(name="cfg3_nt32_p05", ns=768, nt=32, ds=0.6, dt=0.6, npt=1000, pitch=0.5, rot=4.0, nx=256, ny=256, dx=0.5, dz=0.5),
    dict(name="cfg3_nt64_p15", ns=896, nt=64, ds=0.55, dt=0.55, npt=1200, pitch=1.5, rot=3.0, nx=384, ny=384, dx=0.5, dz=0.5),
    # edge cases
    dict(name="small_test", ns=96, nt=8, ds=1.0, dt=1.0, npt=120, pitch=1.0, views=1618, nx=32, ny=32, dx=1.0, dz=1.0),
    dict(name="descending_couch", ns=128, nt=16, ds=0.8, dt=0.8, npt=200, pitch=1.0, rot=12.0, nx=64, ny=64, dx=1.0, dz=0.7, z_dir=-1, z_start=500.0),
    dict(name="wrapped_start", ns=128, nt=16, ds=0.8, dt=0.8, npt=200, pitch=1.2, rot=12.0, nx=64, ny=48, dx=1.1, dz=0.9, start=2 * math.pi - 0.01),
    dict(name="offsets_odd", ns=101, nt=12, ds=0.9, dt=0.7, npt=150, pitch=0.9, rot=14.0, nx=40, ny=56, dx=0.9, dz=0.6, off_x=1.5, off_y=-2.25, cc=49.25, z_start=-123.4),
    dict(name="too_short", ns=128, nt=16, ds=0.8, dt=0.8, npt=200, pitch=1.0, rot=1.5, nx=64, ny=64, dx=1.0, dz=1.0),
]


def case_arrays(c: dict):
    """float32 angles and couch positions of a case (what the files hold)."""
    readings = c.get("views") or int(round(c["rot"] * c["npt"]))
    feed = c["pitch"] * c["nt"] * c["dt"]
    j = np.arange(readings, dtype=np.float64)
    ang = np.mod(c.get("start", 0.0) + j * (2.0 * math.pi / c["npt"]), 2.0 * math.pi)
    z = c.get("z_start", 0.0) + c.get("z_dir", 1) * j * (feed / c["npt"])
    return ang.astype(np.float32), z.astype(np.float32), readings


def case_prm_values(c: dict) -> dict:
    _, _, readings = case_arrays(c)
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    return dict(
        Ns=c["ns"], Nt=c["nt"], Ds=f32(c["ds"]), Dt=f32(c["dt"]),
        PitchValue=f32(c["pitch"] * c["nt"] * c["dt"]), Nx=c["nx"], Ny=c["ny"], Dx=f32(c["dx"]),
        Dz=f32(c["dz"]), OffsetX=f32(c.get("off_x", 0.0)), OffsetY=f32(c.get("off_y", 0.0)),
        Readings=readings, ViewOffset=0, DataOffset=0, RSrcToIso=f32(c.get("dso", 570.0)),
        CentralChannel=f32(c.get("cc", (c["ns"] - 1) / 2.0)), NProjTurn=c["npt"])


def write_case(c: dict, d: Path) -> Path:
    ang, z, _ = case_arrays(c)
    ang.tofile(d / "angles.raw")
    z.tofile(d / "couch.raw")
    (d / "proj.raw").write_bytes(b"\0" * 16)  # ReconData only checks that it opens
    vals = case_prm_values(c)
    lines = [f"RawDataDir: {d}/", "DataInterpFile: proj.raw", "ViewAngleFile: angles.raw",
             "CouchPosFile: couch.raw", f"OutputDir: {d}/", "OutputName: image.raw"]
    lines += [f"{k}: {v!r}" for k, v in vals.items()]
    prm = d / "case.prm"
    prm.write_text("\n".join(lines) + "\n")
    return prm


def main() -> None:
    if not REF_PLAN.exists():
        sys.exit(f"{REF_PLAN} missing: run `make -C oracle ref` with the reference tree present")
    plans = []
    for c in CASES:
        with tempfile.TemporaryDirectory() as td:
            prm = write_case(c, Path(td))
            r = subprocess.run([str(REF_PLAN), "plan", str(prm)], capture_output=True, text=True)
        rec = dict(case=c)
        if r.returncode != 0:
            rec["error"] = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else r.stderr.strip()
        else:
            out = r.stdout[r.stdout.index("{\"ctg\""):]
            rec["ref"] = json.loads(out)
        plans.append(rec)
        print(c["name"], "error" if "error" in rec else f"{rec['ref']['ri']['n_blocks']} blocks")
    (HERE / "plans.json").write_text(json.dumps(plans, indent=1) + "\n")
    taps = []
    for ns, ds in [(96, 1.0), (672, 1.0), (736, 0.6), (896, 0.5), (101, 0.9)]:
        r = subprocess.run([str(REF_PLAN), "taps", str(ns), repr(ds)], capture_output=True,
                           text=True, check=True)
        taps.append(json.loads(r.stdout))
    (HERE / "taps.json").write_text(json.dumps(taps) + "\n")


if __name__ == "__main__":
    main()
