"""ctypes binding of include/lct.h (liblct.so).

The library is loaded from the package directory.  There is no fallback: if liblct.so is
missing or fails to load, every entry point raises, so nothing silently runs elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblct.so"

LCT_OK = 0
LCT_ERR_ARG = 1
LCT_ERR_CUDA = 2
LCT_ERR_ALLOC = 3
LCT_ERR_RANGE = 4
LCT_ERR_DEVICE = 5
LCT_ERR_UNSUPPORTED = 6
LCT_ERR_IO = 7
LCT_ERR_SCRATCH = 8

INTERP_TEX8, INTERP_EXACT = 0, 1
ADDR_BORDER, ADDR_CLAMP, ADDR_LEGACY = 0, 1, 2
FILTER_RAMLAK, FILTER_SHEPP_LOGAN = 0, 1
WINDOW_NONE, WINDOW_HANN, WINDOW_HAMMING, WINDOW_COSINE = 0, 1, 2, 3
FILTER_FP32, FILTER_BF16X3, FILTER_BF16X6 = 0, 1, 2
MODE_BLOCK, MODE_SCAN = 0, 1
REBIN_FAN2PAR, REBIN_NULL, REBIN_PI_ORI = 0, 1, 2
PW_NONE, PW_PI_ORI = 0, 1
BP_PAR, BP_PI_ORI = 0, 1
BP_SAMPLER_AUTO, BP_SAMPLER_QUADS, BP_SAMPLER_TEXTURE, BP_SAMPLER_QUADS_TMA = 0, 1, 2, 3


class LctError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _status_string(status)
        if status == LCT_ERR_CUDA and _lib is not None:
            msg += f" (cudaError {_lib.lct_last_cuda_error()})"
        super().__init__(f"{what}: {msg}" if what else msg)


class Geom(C.Structure):
    """lct_geom == CTGeom (Include/DataStructs.h:15-28)."""

    _fields_ = [
        ("orbit", C.c_float), ("orbit_start", C.c_float),
        ("ns", C.c_int), ("nt", C.c_int),
        ("ws", C.c_float), ("wt", C.c_float),
        ("n_angle", C.c_int), ("n_angle_add", C.c_int),
        ("ds", C.c_float), ("dt", C.c_float),
        ("pitch", C.c_float), ("source_z0", C.c_float), ("dso", C.c_float),
        ("n_proj_turn", C.c_int), ("z_dir", C.c_int), ("add_projections", C.c_int),
    ]


class Img(C.Structure):
    """lct_img == ImgGeom (Include/DataStructs.h:109-115)."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("wx", C.c_float), ("wy", C.c_float), ("wz", C.c_float),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
    ]


class ScanParams(C.Structure):
    _fields_ = [
        ("ns", C.c_int), ("nt", C.c_int), ("ds", C.c_float), ("dt", C.c_float),
        ("pitch_value", C.c_float), ("nx", C.c_int), ("ny", C.c_int),
        ("dx", C.c_float), ("dz", C.c_float), ("offset_x", C.c_float), ("offset_y", C.c_float),
        ("readings", C.c_int), ("view_offset", C.c_int), ("data_offset", C.c_int),
        ("r_src_to_iso", C.c_float), ("central_channel", C.c_float),
        ("n_proj_turn", C.c_int), ("max_blocks", C.c_int), ("first_block", C.c_int),
    ]


class PlanInfo(C.Structure):
    _fields_ = [
        ("ctg", Geom), ("ig", Img),
        ("n_readings", C.c_int),
        ("data_begin_pos", C.c_float), ("data_end_pos", C.c_float),
        ("allow_begin", C.c_float), ("allow_end", C.c_float),
        ("start_pos", C.c_float), ("end_pos", C.c_float),
        ("recon_start_pos", C.c_float), ("recon_end_pos", C.c_float),
        ("n_slices_recon", C.c_int), ("n_slices_block", C.c_int), ("n_blocks", C.c_int),
        ("data_offset", C.c_int), ("first_block", C.c_int), ("n_blocks_run", C.c_int),
    ]


class BlockInfo(C.Structure):
    _fields_ = [
        ("block_idx", C.c_int), ("block_proj_start", C.c_int), ("block_proj_end", C.c_int),
        ("block_start", C.c_float), ("block_end", C.c_float),
        ("block_slice_start", C.c_int), ("block_slice_end", C.c_int),
    ]


class ReconStats(C.Structure):
    _fields_ = [
        ("voxel_updates", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
        ("rebinned_views", C.c_int64), ("launches", C.c_int),
    ]


class ReconOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("rebinner", C.c_int), ("preweight", C.c_int),
        ("filter_kind", C.c_int), ("window", C.c_int), ("filter_mode", C.c_int),
        ("backprojector", C.c_int), ("interp", C.c_int), ("addr", C.c_int), ("bp_nz", C.c_int),
        ("bp_minb", C.c_int), ("bp_sampler", C.c_int),
    ]


P = C.c_void_p
I32 = C.c_int
I64 = C.c_int64
F32 = C.c_float
F64 = C.c_double
U64 = C.c_uint64
GP = C.POINTER(Geom)
IP = C.POINTER(Img)

# name -> (restype, argtypes); every symbol include/lct.h declares
CNN_TRAIN = 1

SIGNATURES: dict[str, tuple] = {
    "lct_status_string": (C.c_char_p, [I32]),
    "lct_last_cuda_error": (I32, []),
    "lct_device_status": (I32, [C.POINTER(I32)]),
    "lct_version": (I32, []),
    "lct_rebin_fan2par": (I32, [GP, P, P, I32, I32, P]),
    "lct_rebin_fan2par_index": (I32, [GP, I32, P, P, P]),
    "lct_rebin_fan2par_scan": (I32, [GP, P, I64, I64, P, I64, I64, I32, I32, I32, P]),
    "lct_rebin_null": (I32, [GP, P, P, I32, P]),
    "lct_rebin_pi_ori": (I32, [GP, P, P, I32, I32, P]),
    "lct_weight_pi_ori": (I32, [GP, P, P]),
    "lct_filter_taps": (I32, [I32, I32, I32, F32, P]),
    "lct_filter_rows": (I32, [I32, P, P, I64, I32, P]),
    "lct_backproject_par": (I32, [GP, IP, P, P, P, I32, I32, P]),
    "lct_backproject_par_noalloc": (I32, [GP, IP, P, P, P, I32, I32, P]),
    "lct_backproject_par_quad_path": (I32, [GP, IP, C.POINTER(I32)]),
    "lct_backproject_pi_ori": (I32, [GP, IP, P, P, P, I32, I32, P]),
    "lct_plan_create": (I32, [C.POINTER(ScanParams), P, P, C.POINTER(P)]),
    "lct_plan_adopt": (I32, [C.POINTER(PlanInfo), C.POINTER(BlockInfo), I32, P, P, C.POINTER(P)]),
    "lct_plan_info_get": (I32, [P, C.POINTER(PlanInfo)]),
    "lct_plan_block": (I32, [P, I32, C.POINTER(BlockInfo)]),
    "lct_plan_destroy": (None, [P]),
    "lct_recon_opts_default": (None, [C.POINTER(ReconOpts)]),
    "lct_recon_create": (I32, [P, C.POINTER(ReconOpts), C.POINTER(P)]),
    "lct_recon_create_bounded": (I32, [P, C.POINTER(ReconOpts), I32, C.POINTER(P)]),
    "lct_recon_device_bytes": (I32, [P, C.POINTER(I64)]),
    "lct_recon_run_file": (I32, [P, C.c_char_p, C.c_char_p, P, P]),
    "lct_recon_run": (I32, [P, P, I64, I32, P, I32, P]),
    "lct_recon_last_times": (I32, [P, P]),
    "lct_recon_io_times": (I32, [P, P]),
    "lct_recon_fan_range": (I32, [P, C.POINTER(I64), C.POINTER(I64)]),
    "lct_recon_stats_get": (I32, [P, C.POINTER(ReconStats)]),
    "lct_recon_destroy": (None, [P]),
    "lct_recon_autotune": (I32, [P, C.POINTER(I32), C.POINTER(I32)]),
    "lct_batch_create": (I32, [P, I32, C.POINTER(ReconOpts), C.POINTER(P)]),
    "lct_batch_run": (I32, [P, P, P, I32, P, I32, P]),
    "lct_batch_fan_range": (I32, [P, I32, C.POINTER(I64), C.POINTER(I64)]),
    "lct_batch_stats_get": (I32, [P, C.POINTER(ReconStats)]),
    "lct_batch_last_times": (I32, [P, P]),
    "lct_batch_destroy": (None, [P]),
    "lct_sim_project": (I32, [P, I32, I32, I32, F32, F32, F32, F32, F32, P, P, I64, I64, F64, U64, P, P]),
    "lct_voxelise": (I32, [P, I32, I32, I32, I32, F64, F64, F64, F64, F64, F64, I32, P, P]),
    "lct_cnn_param_count": (I32, [P]),
    "lct_cnn_create": (I32, [I32, I32, I32, I32, U64, P]),
    "lct_cnn_set_params": (I32, [P, P, I32]),
    "lct_cnn_get_params": (I32, [P, P, I32]),
    "lct_cnn_get_grads": (I32, [P, P, I32]),
    "lct_cnn_set_scales": (I32, [P, F32, F32]),
    "lct_cnn_get_scales": (I32, [P, P, P]),
    "lct_cnn_forward": (I32, [P, P, I32, P, P]),
    "lct_cnn_backward": (I32, [P, P, P, I32, P]),
    "lct_cnn_adam_step": (I32, [P, F32, F32, F32, F32, P]),
    "lct_cnn_train_step": (I32, [P, P, P, I32, F32, P]),
    "lct_cnn_last_loss": (I32, [P, P]),
    "lct_cnn_infer_volume": (I32, [P, P, P, I32, F32, P, P]),
    "lct_cnn_last_rejected": (I32, [P, P]),
    "lct_cnn_get_shape": (I32, [P, P, P, P]),
    "lct_cnn_destroy": (None, [P]),
    "lct_recon_set_learned": (I32, [P, P, F32]),
    "lct_recon_learned_info": (I32, [P, P, P]),
}

_lib: C.CDLL | None = None


def _status_string(status: int) -> str:
    if _lib is None:
        return f"status {status}"
    return _lib.lct_status_string(status).decode()


def load() -> C.CDLL:
    """Load liblct.so (raises if it is missing: there is no other implementation)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m listctrecons_b200.build`")
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def lib() -> C.CDLL:
    return load()


PROBE_PATH = Path(__file__).resolve().parent / "liblctprobe.so"
_probe = None


def load_probe() -> C.CDLL:
    """liblctprobe.so: measurement probes (texture-unit samples, L1 load bandwidth) used by the
    tests and the benchmark; nothing in liblct.so depends on it.  Functions return 0 or a
    cudaError_t value."""
    global _probe
    if _probe is None:
        if not PROBE_PATH.exists():
            raise ImportError(f"{PROBE_PATH} is missing: build it with `python -m listctrecons_b200.build`")
        p = C.CDLL(os.fspath(PROBE_PATH))
        p.lctp_tex3d_sample.restype = I32
        p.lctp_tex3d_sample.argtypes = [P, I32, I32, I32, P, I64, I32, P]
        p.lctp_l1_load_gbs.restype = I32
        p.lctp_l1_load_gbs.argtypes = [I32, I32, I32, C.POINTER(F64), C.POINTER(F64)]
        _probe = p
    return _probe


def check(status: int, what: str = "") -> None:
    if status != LCT_OK:
        raise LctError(status, what)


def declared_symbols() -> list[str]:
    """Function names declared in include/lct.h (parsed from the header)."""
    import re

    hdr = (Path(__file__).resolve().parent.parent / "include" / "lct.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(lct_[a-z0-9_]+)\s*\(", hdr)))
