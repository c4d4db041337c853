"""Helical scans for the reconstruction: geometry, seeded ellipsoid phantoms, simulation on the
GPU, and the reference's file formats.

Geometry mapping (a scanner description -> the reference's .prm keys):
  RSrcToIso = source-to-iso distance; Ds/Dt = column/row spacing at iso; CentralChannel =
  (ns-1)/2; PitchValue = table feed per rotation = pitch * nt * dt; Dx = voxel size (dy = dx);
  Dz = slice spacing; Readings = number of views; ViewOffset = DataOffset = 0.
  View angles b_j = start + j 2 pi / npt wrapped to [0, 2 pi), couch z_j = z_start + dir j feed /
  npt.  FP64 copies are kept; the files hold float32, as the reference reads them
  (Src/DataStructs.cpp:138-160).  The source-detector distance does not enter the reference
  algorithm (Ds and Dt are at iso) and is not needed.

Phantoms: seeded random ellipsoids (numpy PCG64).  Densities in [0, 2] are scaled by
mu_water = 0.02 / mm to attenuation so exp(-p) stays representable through 80-mm semi-axes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import capi
from .prm import FileParams

MU_WATER = 0.02  # 1/mm


@dataclass
class ScanGeometry:
    ns: int
    nt: int
    ds: float            # mm at iso
    dt: float            # mm at iso
    npt: int             # views per rotation
    pitch: float         # helical pitch (feed / (nt * dt))
    nx: int
    ny: int
    dx: float
    dz: float
    dso: float = 570.0
    readings: int = 0
    start_angle: float = 0.0
    z_start: float = 0.0
    z_dir: int = 1
    offset_x: float = 0.0
    offset_y: float = 0.0
    max_blocks: int = 0

    @property
    def feed(self) -> float:
        return self.pitch * self.nt * self.dt

    @property
    def central_channel(self) -> float:
        return (self.ns - 1) / 2.0

    def angles64(self) -> np.ndarray:
        j = np.arange(self.readings, dtype=np.float64)
        return np.mod(self.start_angle + j * (2.0 * math.pi / self.npt), 2.0 * math.pi)

    def zpos64(self) -> np.ndarray:
        j = np.arange(self.readings, dtype=np.float64)
        return self.z_start + self.z_dir * j * (self.feed / self.npt)

    def angles32(self) -> np.ndarray:
        return self.angles64().astype(np.float32)

    def zpos32(self) -> np.ndarray:
        return self.zpos64().astype(np.float32)

    def scan_params(self) -> capi.ScanParams:
        p = capi.ScanParams()
        p.ns, p.nt, p.ds, p.dt = self.ns, self.nt, self.ds, self.dt
        p.pitch_value = np.float32(self.feed)
        p.nx, p.ny, p.dx, p.dz = self.nx, self.ny, self.dx, self.dz
        p.offset_x, p.offset_y = self.offset_x, self.offset_y
        p.readings, p.view_offset, p.data_offset = self.readings, 0, 0
        p.r_src_to_iso = self.dso
        p.central_channel = self.central_channel
        p.n_proj_turn = self.npt
        p.max_blocks = self.max_blocks
        return p

    def file_params(self, data_dir: str, out_dir: str, out_name: str = "image.raw") -> FileParams:
        d = data_dir.rstrip("/") + "/"
        o = out_dir.rstrip("/") + "/"

        def f32(v):  # decimal that parses to exactly the float the planner is given
            return float(np.float32(v))

        return FileParams(
            RawDataDir=d, DataInterpFile="proj.raw", ViewAngleFile="angles.raw",
            CouchPosFile="couch.raw", OutputDir=o, OutputName=out_name,
            Ns=self.ns, Nt=self.nt, Ds=f32(self.ds), Dt=f32(self.dt), PitchValue=f32(self.feed),
            Nx=self.nx, Ny=self.ny, Dx=f32(self.dx), Dz=f32(self.dz), OffsetX=f32(self.offset_x),
            OffsetY=f32(self.offset_y), Readings=self.readings, ViewOffset=0, DataOffset=0,
            RSrcToIso=f32(self.dso), CentralChannel=f32(self.central_channel),
            NProjTurn=self.npt, MaxBlocks=self.max_blocks)

    def with_blocks(self, nblocks: int, cap: bool = True) -> "ScanGeometry":
        """Smallest number of views for which the planner plans >= nblocks blocks (the
        reference has no z-range key, so scan length decides the slice count); with cap,
        MaxBlocks is set so exactly nblocks are reconstructed."""
        from .recon import Plan

        g = ScanGeometry(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        g.max_blocks = 0
        lo, hi = 101, 101
        while True:
            g.readings = hi
            try:
                if Plan(g).info.n_blocks >= nblocks:
                    break
            except capi.LctError:
                pass
            lo, hi = hi, hi * 2
            if hi > 10_000_000:
                raise ValueError("geometry never reaches the requested block count")
        while hi - lo > 1:
            mid = (lo + hi) // 2
            g.readings = mid
            try:
                ok = Plan(g).info.n_blocks >= nblocks
            except capi.LctError:
                ok = False
            if ok:
                hi = mid
            else:
                lo = mid
        g.readings = hi
        if cap:
            g.max_blocks = nblocks
        return g


# ------------------------------------------------------------------------------------------
# phantoms
# ------------------------------------------------------------------------------------------
def _rotation(phi: float, theta: float, psi: float) -> np.ndarray:
    """Rz(phi) Ry(theta) Rz(psi): ellipsoid frame -> world."""
    def rz(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], dtype=np.float64)

    def ry(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], dtype=np.float64)

    return rz(phi) @ ry(theta) @ rz(psi)


@dataclass
class Phantom:
    """Ellipsoid records, 16 doubles each: centre(3), semi-axes(3), rotation(9), mu."""

    records: np.ndarray = field(default_factory=lambda: np.zeros((0, 16)))

    @classmethod
    def random(cls, n: int, seed: int, fov_radius: float, z_lo: float, z_hi: float,
               semi=(5.0, 80.0), density=(0.0, 2.0), mu_water: float = MU_WATER) -> "Phantom":
        rng = np.random.Generator(np.random.PCG64(seed))
        recs = np.zeros((n, 16), dtype=np.float64)
        for m in range(n):
            ax, ay, az = rng.uniform(semi[0], semi[1], size=3)
            ax, ay = min(ax, 0.9 * fov_radius), min(ay, 0.9 * fov_radius)
            r = rng.uniform(0.0, max(fov_radius - max(ax, ay), 0.0))
            a = rng.uniform(0.0, 2 * math.pi)
            cz = rng.uniform(z_lo, z_hi)
            R = _rotation(*rng.uniform(0.0, 2 * math.pi, size=3))
            mu = rng.uniform(density[0], density[1]) * mu_water
            recs[m, 0:3] = (r * math.cos(a), r * math.sin(a), cz)
            recs[m, 3:6] = (ax, ay, az)
            recs[m, 6:15] = R.reshape(-1)
            recs[m, 15] = mu
        return cls(recs)

    @classmethod
    def head_like(cls, seed: int, fov_radius: float, z_lo: float, z_hi: float) -> "Phantom":
        """A seeded nested-ellipsoid phantom: an outer shell, an inner filling and a few small
        features (a stand-in for the 3-D Shepp-Logan table, which is not available offline)."""
        rng = np.random.Generator(np.random.PCG64(seed))
        zc = 0.5 * (z_lo + z_hi)
        hz = max(0.5 * (z_hi - z_lo), 10.0)
        R0 = fov_radius * 0.85
        recs = [
            (0, 0, zc, R0 * 0.92, R0, hz * 1.5, 0.0, 2.0 * MU_WATER),
            (0, -R0 * 0.02, zc, R0 * 0.87, R0 * 0.94, hz * 1.45, 0.0, -1.0 * MU_WATER),
        ]
        for _ in range(8):
            ax, ay, az = rng.uniform(0.05, 0.25, size=3) * R0
            r = rng.uniform(0, 0.55 * R0)
            a = rng.uniform(0, 2 * math.pi)
            recs.append((r * math.cos(a), r * math.sin(a), zc + rng.uniform(-0.5, 0.5) * hz,
                         ax, ay, az * 1.5, rng.uniform(0, math.pi),
                         rng.uniform(-0.2, 0.3) * MU_WATER))
        out = np.zeros((len(recs), 16))
        for m, (x, y, z, ax, ay, az, phi, mu) in enumerate(recs):
            out[m, 0:3] = (x, y, z)
            out[m, 3:6] = (ax, ay, az)
            out[m, 6:15] = _rotation(phi, 0.0, 0.0).reshape(-1)
            out[m, 15] = mu
        return cls(out)


# ------------------------------------------------------------------------------------------
# simulation on the GPU and the reference's files
# ------------------------------------------------------------------------------------------
def simulate_gpu(geo: ScanGeometry, phantom: Phantom, i0: float = 1e5, seed: int = 1,
                 v0: int = 0, v1: int | None = None, out=None):
    """Fan projections [v1-v0][nt][ns] float32 as a CUDA torch tensor (lct_sim_project)."""
    import torch

    lib = capi.load()
    v1 = geo.readings if v1 is None else v1
    dev = torch.device("cuda")
    ell = torch.as_tensor(np.ascontiguousarray(phantom.records), dtype=torch.float64, device=dev)
    ang = torch.as_tensor(geo.angles64(), device=dev)
    zp = torch.as_tensor(geo.zpos64(), device=dev)
    if out is None:
        out = torch.empty((v1 - v0, geo.nt, geo.ns), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    capi.check(lib.lct_sim_project(ell.data_ptr(), len(phantom.records), geo.ns, geo.nt, geo.ds,
                                   geo.dt, np.float32(geo.central_channel),
                                   np.float32((geo.nt - 1) / 2.0), geo.dso, ang.data_ptr(),
                                   zp.data_ptr(), v0, v1, float(i0), int(seed), out.data_ptr(),
                                   stream), "lct_sim_project")
    return out


def write_scan_files(geo: ScanGeometry, fan: np.ndarray, data_dir: str | Path, out_dir: str | Path,
                     prm_name: str = "scan.prm") -> Path:
    """Writes proj.raw, angles.raw, couch.raw and the .prm (reference formats)."""
    data_dir, out_dir = Path(data_dir), Path(out_dir)
    data_dir.mkdir(parents=True, exist_ok=True)
    out_dir.mkdir(parents=True, exist_ok=True)
    np.ascontiguousarray(fan, dtype=np.float32).tofile(data_dir / "proj.raw")
    geo.angles32().tofile(data_dir / "angles.raw")
    geo.zpos32().tofile(data_dir / "couch.raw")
    prm = data_dir / prm_name
    geo.file_params(str(data_dir), str(out_dir)).write(prm)
    return prm
