"""TEST INFRASTRUCTURE ONLY: Python access to the CPU oracle (fdk_oracle.c -> liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and
only as the checker / the timed CPU restatement -- never as the thing measured or shipped.
It is independent of the product package (its own struct definitions).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

EXACT, TEXEMU = 0, 1
BORDER, CLAMP = 0, 1
Q_NEAREST, Q_TRUNC = 0, 1


class Geom(C.Structure):  # CTGeom, Include/DataStructs.h:15-28
    _fields_ = [
        ("orbit", C.c_float), ("orbit_start", C.c_float), ("ns", C.c_int), ("nt", C.c_int),
        ("ws", C.c_float), ("wt", C.c_float), ("n_angle", C.c_int), ("n_angle_add", C.c_int),
        ("ds", C.c_float), ("dt", C.c_float), ("pitch", C.c_float), ("source_z0", C.c_float),
        ("dso", C.c_float), ("n_proj_turn", C.c_int), ("z_dir", C.c_int),
        ("add_projections", C.c_int),
    ]


class Img(C.Structure):  # ImgGeom, Include/DataStructs.h:109-115
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("wx", C.c_float), ("wy", C.c_float),
        ("wz", C.c_float), ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
    ]


def build() -> Path:
    """make -C oracle (liboracle.so); also oracle/_ref when the reference tree is present."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(os.fspath(LIB))
        P = C.c_void_p
        G = C.POINTER(Geom)
        Ip = C.POINTER(Img)
        sig = {
            "orc_set_tex_quant": (None, [C.c_int]),
            "orc_get_tex_quant": (C.c_int, []),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_tex3d_sample": (None, [P, C.c_int, C.c_int, C.c_int, P, C.c_long, C.c_int, C.c_int, P]),
            "orc_rebin_fan2par_index": (None, [G, C.c_int, P, P]),
            "orc_rebin_fan2par": (None, [G, P, P, C.c_int, C.c_int]),
            "orc_rebin_null": (None, [G, P, P, C.c_int]),
            "orc_rebin_pi_ori": (None, [G, P, P, C.c_int, C.c_int]),
            "orc_rebin_pi_ori_coords": (None, [G, P]),
            "orc_weight_pi_ori": (None, [G, P]),
            "orc_ramp_taps": (None, [C.c_int, C.c_float, P]),
            "orc_shepp_logan_taps": (None, [C.c_int, C.c_float, P]),
            "orc_filter_rows": (None, [P, C.c_int, P, P, C.c_long, C.c_int]),
            "orc_bp_window": (None, [G, Ip, C.c_int, C.c_float, C.c_int, P, P]),
            "orc_bp_par_rows": (None, [G, Ip, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_bp_par": (None, [G, Ip, P, P, P, C.c_int, C.c_int]),
            "orc_bp_par_cols": (None, [G, Ip, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_bp_pi_ori": (None, [G, Ip, P, P, P, C.c_int, C.c_int]),
            "orc_bp_par_rows_f32": (None, [G, Ip, P, P, P, C.c_int, C.c_int]),
            "orc_rebin_filter_f32": (None, [G, P, P, P, C.c_int, C.c_int]),
            "orc_sim_project": (None, [P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                       C.c_float, C.c_float, P, P, C.c_long, C.c_long, C.c_double,
                                       C.c_uint64, P]),
            "orc_voxelise": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, P]),
            "orc_cnn_param_count": (C.c_int, []),
            "orc_cnn_forward": (None, [P, P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, P]),
            "orc_cnn_loss_grad": (C.c_double, [P, P, P, C.c_int, C.c_int, C.c_int, C.c_float,
                                               C.c_float, C.c_int, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype, f.argtypes = res, args
    return _lib


def geom_from(obj) -> Geom:
    g = Geom()
    for name, _ in Geom._fields_:
        setattr(g, name, getattr(obj, name))
    return g


def img_from(obj) -> Img:
    i = Img()
    for name, _ in Img._fields_:
        setattr(i, name, getattr(obj, name))
    return i


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def set_tex_quant(q: int) -> None:
    lib().orc_set_tex_quant(q)


def tex3d_sample(vol, coords, interp=TEXEMU, addr=BORDER):
    vol = _f32(vol)
    nz, ny, nx = vol.shape
    c = _f32(coords).reshape(-1, 3)
    out = np.zeros(len(c), dtype=np.float64)
    lib().orc_tex3d_sample(vol.ctypes.data, nx, ny, nz, c.ctypes.data, len(c), interp, addr, out.ctypes.data)
    return out


def rebin_fan2par_index(g, interp=TEXEMU):
    idx = np.zeros((g.n_angle, g.ns), dtype=np.int32)
    w = np.zeros((g.n_angle, g.ns), dtype=np.float32)
    lib().orc_rebin_fan2par_index(C.byref(geom_from(g)), interp, idx.ctypes.data, w.ctypes.data)
    return idx, w


def rebin_fan2par(g, fan, interp=TEXEMU, addr=BORDER):
    fan = _f32(fan)
    out = np.zeros((g.n_angle, g.nt, g.ns), dtype=np.float64)
    lib().orc_rebin_fan2par(C.byref(geom_from(g)), fan.ctypes.data, out.ctypes.data, interp, addr)
    return out


def rebin_null(g, fan, addr=BORDER):
    fan = _f32(fan)
    out = np.zeros((g.n_angle, g.nt, g.ns), dtype=np.float64)
    lib().orc_rebin_null(C.byref(geom_from(g)), fan.ctypes.data, out.ctypes.data, addr)
    return out


def rebin_pi_ori(g, fan, interp=TEXEMU, addr=BORDER):
    fan = _f32(fan)
    out = np.zeros((g.n_angle, g.nt, g.ns), dtype=np.float64)
    lib().orc_rebin_pi_ori(C.byref(geom_from(g)), fan.ctypes.data, out.ctypes.data, interp, addr)
    return out


def rebin_pi_ori_coords(g):
    """[n_angle][nt][ns][3] float32 texture coordinates the reference's PI-original rebin samples
    at (CUDA/Rebiner.cu:156-179, its FP32 expressions)."""
    out = np.zeros((g.n_angle, g.nt, g.ns, 3), dtype=np.float32)
    lib().orc_rebin_pi_ori_coords(C.byref(geom_from(g)), out.ctypes.data)
    return out


def weight_pi_ori(g, proj):
    out = np.array(proj, dtype=np.float64, copy=True, order="C")
    lib().orc_weight_pi_ori(C.byref(geom_from(g)), out.ctypes.data)
    return out


def ramp_taps(ns, ds):
    h = np.zeros(2 * ns, dtype=np.float32)
    lib().orc_ramp_taps(ns, ds, h.ctypes.data)
    return h


def shepp_logan_taps(ns, ds):
    h = np.zeros(2 * ns, dtype=np.float32)
    lib().orc_shepp_logan_taps(ns, ds, h.ctypes.data)
    return h


def filter_rows(h, rows, mode=0):
    """mode 0: FP64 sums; mode 1: FP32 FMA in the reference's order."""
    rows = _f32(rows)
    ns = rows.shape[-1]
    out = np.zeros(rows.shape, dtype=np.float64)
    lib().orc_filter_rows(_f32(h).ctypes.data, ns, rows.ctypes.data, out.ctypes.data,
                          rows.size // ns, mode)
    return out


def bp_window(g, ig, iz):
    a, b = C.c_int(), C.c_int()
    dzv = np.float32(np.float32(g.pitch) / np.float32(g.n_proj_turn))
    lib().orc_bp_window(C.byref(geom_from(g)), C.byref(img_from(ig)), iz, float(dzv),
                        g.n_proj_turn // 2, C.byref(a), C.byref(b))
    return a.value, b.value


def bp_par(g, ig, betas, proj, interp=TEXEMU, addr=BORDER, rows=None):
    proj = _f32(proj)
    b = _f32(betas)
    img = np.zeros((ig.nz, ig.ny, ig.nx), dtype=np.float64)
    y0, y1 = (0, ig.ny) if rows is None else rows
    lib().orc_bp_par_rows(C.byref(geom_from(g)), C.byref(img_from(ig)), b.ctypes.data,
                          proj.ctypes.data, img.ctypes.data, interp, addr, y0, y1)
    return img


def bp_par_cols(g, ig, betas, proj, interp=TEXEMU, addr=BORDER, rows=None, ystep=1):
    """bp_par with the loops interchanged (z-invariant terms once per voxel column and view):
    bit-identical to bp_par and several times faster; used for whole-slab checks.  Rows
    y0, y0 + ystep, ... below y1 are computed, the others stay 0."""
    proj = _f32(proj)
    b = _f32(betas)
    img = np.zeros((ig.nz, ig.ny, ig.nx), dtype=np.float64)
    y0, y1 = (0, ig.ny) if rows is None else rows
    lib().orc_bp_par_cols(C.byref(geom_from(g)), C.byref(img_from(ig)), b.ctypes.data,
                          proj.ctypes.data, img.ctypes.data, interp, addr, y0, y1, ystep)
    return img


def filter_rows_fp64(h, rows):
    """filter_rows mode 0 as one FP64 matrix product with the Toeplitz matrix
    T[k][n] = h[n - k + ns] (CUDA/Filter.cu:42-46): the same sums in another order, within
    1e-14 relative of filter_rows; used for whole-slab checks."""
    rows = _f32(rows)
    ns = rows.shape[-1]
    k = np.arange(ns)
    T = np.asarray(h, dtype=np.float32).astype(np.float64)[k[None, :] - k[:, None] + ns]
    return (rows.reshape(-1, ns).astype(np.float64) @ T).reshape(rows.shape)


def bp_pi_ori(g, ig, betas, proj, interp=EXACT, addr=BORDER):
    proj = _f32(proj)
    b = _f32(betas)
    img = np.zeros((ig.nz, ig.ny, ig.nx), dtype=np.float64)
    lib().orc_bp_pi_ori(C.byref(geom_from(g)), C.byref(img_from(ig)), b.ctypes.data,
                        proj.ctypes.data, img.ctypes.data, interp, addr)
    return img


def bp_par_rows_f32(g, ig, betas, proj, y0, y1, out=None):
    proj = _f32(proj)
    b = _f32(betas)
    img = out if out is not None else np.zeros((ig.nz, ig.ny, ig.nx), dtype=np.float32)
    lib().orc_bp_par_rows_f32(C.byref(geom_from(g)), C.byref(img_from(ig)), b.ctypes.data,
                              proj.ctypes.data, img.ctypes.data, y0, y1)
    return img


def rebin_filter_f32(g, fan, h, v0, v1):
    fan = _f32(fan)
    out = np.zeros((v1 - v0, g.nt, g.ns), dtype=np.float32)
    lib().orc_rebin_filter_f32(C.byref(geom_from(g)), fan.ctypes.data, _f32(h).ctypes.data,
                               out.ctypes.data, v0, v1)
    return out


def sim_project(ellipsoids, ns, nt, ds, dt, ws, wt, dso, angles64, zpos64, v0, v1, i0, seed):
    e = np.ascontiguousarray(ellipsoids, dtype=np.float64)
    a = np.ascontiguousarray(angles64, dtype=np.float64)
    z = np.ascontiguousarray(zpos64, dtype=np.float64)
    out = np.zeros((v1 - v0, nt, ns), dtype=np.float32)
    lib().orc_sim_project(e.ctypes.data, len(e), ns, nt, ds, dt, ws, wt, dso, a.ctypes.data,
                          z.ctypes.data, v0, v1, float(i0), int(seed), out.ctypes.data)
    return out


def voxelise(ellipsoids, nx, ny, nz, x0, y0, z0, dx, dy, dz, ss=4):
    e = np.ascontiguousarray(ellipsoids, dtype=np.float64)
    out = np.zeros((nz, ny, nx), dtype=np.float32)
    lib().orc_voxelise(e.ctypes.data, len(e), nx, ny, nz, x0, y0, z0, dx, dy, dz, ss, out.ctypes.data)
    return out


# ------------------------------------------------------------------------------------------
# learned correction (cnn_oracle.c)
# ------------------------------------------------------------------------------------------
CNN_CIN = (5, 32, 32, 32, 32, 32, 32, 32)
CNN_COUT = (32, 32, 32, 32, 32, 32, 32, 1)


def cnn_param_count() -> int:
    return lib().orc_cnn_param_count()


def cnn_forward(params, in5, k_in: float, bf16: bool = True) -> np.ndarray:
    """Residual r [B][H][W] (network units) for 5-slice inputs in5 [B][5][H][W]."""
    p = np.ascontiguousarray(params, dtype=np.float64)
    x = _f32(in5)
    B, _, H, W = x.shape
    r = np.zeros((B, H, W), dtype=np.float64)
    lib().orc_cnn_forward(p.ctypes.data, x.ctypes.data, B, H, W, float(k_in), int(bf16), r.ctypes.data)
    return r


def cnn_loss_grad(params, in5, target, k_in: float, s: float, bf16: bool = True):
    """(loss, gradient) of mean((k_in x_c + r - s t)^2) with respect to the parameters."""
    p = np.ascontiguousarray(params, dtype=np.float64)
    x, t = _f32(in5), _f32(target)
    B, _, H, W = x.shape
    g = np.zeros_like(p)
    loss = lib().orc_cnn_loss_grad(p.ctypes.data, x.ctypes.data, t.ctypes.data, B, H, W,
                                   float(k_in), float(s), int(bf16), g.ctypes.data)
    return loss, g


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))
