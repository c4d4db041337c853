"""Generates the GPU-derived golden fixtures (run on a B200, outputs committed):

  tex_hw.npz         samples of the texture unit's linear filter (cudaFilterModeLinear through
                     lctp_tex3d_sample in liblctprobe.so): a 1-D weight sweep and random 2-D bilinear samples
                     (z at a texel centre, the backprojector's case) with their volume;
  ref_gpu_small.npz  the reference program's own CUDA path (oracle/_ref/ref_timed, built from
                     the reference sources) on a small helical scan simulated by the CPU oracle:
                     its reconstructed image and the head of its filtered block (rebin.raw).

The scan input is regenerated bit for bit by the CPU tests from the parameters in
`small_scan()` with the oracle's simulator, so only the outputs are stored.

    python tests/golden/make_gpu_golden.py OUTDIR
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def small_scan():
    """(geometry, phantom, fan) of the golden scan; fan from the CPU oracle's simulator."""
    import oracle as orc
    from listctrecons_b200.scan import Phantom, ScanGeometry
    from listctrecons_b200.recon import Plan

    geo = ScanGeometry(ns=96, nt=8, ds=1.0, dt=1.0, npt=120, pitch=1.0, nx=32, ny=32, dx=1.0,
                       dz=1.0).with_blocks(2, cap=False)
    p = Plan(geo)
    ph = Phantom.random(6, seed=3, fov_radius=14.0, z_lo=p.blocks[0].block_start,
                        z_hi=p.blocks[-1].block_end, semi=(2.0, 9.0))
    fan = orc.sim_project(ph.records, geo.ns, geo.nt, geo.ds, geo.dt,
                          np.float32(geo.central_channel), np.float32((geo.nt - 1) / 2.0),
                          geo.dso, geo.angles64(), geo.zpos64(), 0, geo.readings, 1e5, 9)
    return geo, ph, fan


def tex_samples():
    from listctrecons_b200 import capi

    probe = capi.load_probe()

    def hw(vol, coords):
        vol = np.ascontiguousarray(vol, np.float32)
        c = np.ascontiguousarray(coords, np.float32)
        out = np.zeros(len(c), np.float32)
        nz, ny, nx = vol.shape
        rc = probe.lctp_tex3d_sample(vol.ctypes.data, nx, ny, nz, c.ctypes.data, len(c), 0,
                                     out.ctypes.data)
        assert rc == 0, f"cudaError {rc}"
        return out

    rng = np.random.default_rng(2024)
    n = 64
    ramp = np.tile(np.arange(n, dtype=np.float32), (2, 2, 1))
    x = np.concatenate([rng.uniform(0.5, n - 1.5, 3000),
                        10.5 + np.arange(1, 1025) / 1024.0]).astype(np.float32)
    c1 = np.stack([x, np.full_like(x, 0.5), np.full_like(x, 0.5)], 1)
    vol2 = rng.uniform(-1, 1, (4, 24, 24)).astype(np.float32)
    m = 4000
    c2 = np.stack([rng.uniform(-0.8, 24.8, m), rng.uniform(-0.8, 24.8, m),
                   rng.integers(0, 4, m) + 0.5], 1).astype(np.float32)
    return dict(ramp_x=x, ramp_hw=hw(ramp, c1), bil_vol=vol2, bil_coord=c2, bil_hw=hw(vol2, c2))


def ref_run(out: Path):
    from listctrecons_b200.scan import write_scan_files

    ref = ROOT / "oracle" / "_ref" / "ref_timed"
    geo, _, fan = small_scan()
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        prm = write_scan_files(geo, fan, td / "data", td / "out")
        r = subprocess.run([str(ref), str(prm)], capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
        img = np.fromfile(td / "out" / "image.raw", dtype=np.float32)
        reb = np.fromfile(td / "out" / "rebin.raw", dtype=np.float32)
    head = reb[: 16 * geo.nt * geo.ns]
    np.savez_compressed(out / "ref_gpu_small.npz", image=img, rebin_head=head)


def main() -> None:
    out = Path(sys.argv[1] if len(sys.argv) > 1 else ".")
    out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out / "tex_hw.npz", **tex_samples())
    ref_run(out)
    print("written", out)


if __name__ == "__main__":
    main()
