"""Host side of the FDK path: the planner, the whole-scan reconstruction, and a mirror of the
reference's stage interfaces over the C ABI.

Mirror of the reference's classes (same names, argument meaning and error behaviour):
  ReconData                 Include/DataStructs.h:313-340 (planner = lct_plan_create)
  GPUMemoryCtrl             Include/GPUMemoryCtrl.h:6-62 (single allocation, bool results)
  Rebiner and subclasses    Include/Rebiner.h:5-35        -> lct_rebin_*
  PreWeighting and subclasses Include/PreWeighting.h:5-27 -> lct_weight_pi_ori (NULL: no-op)
  Filter / RampFilterGPU    Include/Filter.h:5-24         -> lct_filter_taps + lct_filter_rows
  Backprojector and subclasses Include/Backprojector.h:7-28 -> lct_backproject_*
  RawDataReader, RawImageWriter Src/DataReader.cpp, Src/ImageWriter.cpp
  FDKReconstructor          Src/Reconstructor.cpp:11-49
  ReconstrctorAbstractFactory Src/ReconstructorAbstractFactory.cpp:11-33 (misspelling kept)
Device memory comes from torch (plumbing only); every kernel is liblct's.

The B200 path proper is `Reconstruction` (lct_recon_*): all device buffers allocated once,
each view rebinned and filtered once (scan mode), every slab backprojected in one launch.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import capi
from .prm import FileParams, ParameterError

BLOCK_SLICES = 32  # Include/Common.h:4


def _torch():
    import torch

    return torch


def _stream():
    return _torch().cuda.current_stream().cuda_stream


# ------------------------------------------------------------------------------------------
# planner
# ------------------------------------------------------------------------------------------
class Plan:
    """lct_plan: the reference planner's result for one scan (CPU only, no GPU needed)."""

    def __init__(self, geo=None, *, params: capi.ScanParams | None = None,
                 angles32: np.ndarray | None = None, zpos32: np.ndarray | None = None):
        self._lib = capi.load()
        if geo is not None:
            params = geo.scan_params()
            angles32 = geo.angles32()
            zpos32 = geo.zpos32()
        a = np.ascontiguousarray(angles32, dtype=np.float32)
        z = np.ascontiguousarray(zpos32, dtype=np.float32)
        if a.size < params.readings or z.size < params.readings:
            raise ValueError("angle/couch arrays shorter than Readings")
        self.params = params
        self.angles32, self.zpos32 = a, z
        h = C.c_void_p()
        capi.check(self._lib.lct_plan_create(C.byref(params), a.ctypes.data, z.ctypes.data,
                                             C.byref(h)), "lct_plan_create")
        self._h = h
        self.info = capi.PlanInfo()
        capi.check(self._lib.lct_plan_info_get(h, C.byref(self.info)))
        self.blocks = []
        for b in range(self.info.n_blocks):
            bi = capi.BlockInfo()
            capi.check(self._lib.lct_plan_block(h, b, C.byref(bi)))
            self.blocks.append(bi)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.lct_plan_destroy(h)
            self._h = None


def recon_opts(**kw) -> capi.ReconOpts:
    o = capi.ReconOpts()
    capi.load().lct_recon_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


class Reconstruction:
    """lct_recon: device buffers sized from the plan, allocated once; run() reconstructs
    n_blocks_run blocks from host or device fan projections of the whole scan.

    bounded=True: lct_recon_create_bounded -- fan, filtered and quad views in rings sized to the
    slab windows in flight and a four-slab volume ring for host output, so the device footprint
    does not grow with the scan (piece_views: views per rebin/filter/pack step, 0 = default)."""

    def __init__(self, plan: Plan, bounded: bool = False, piece_views: int = 0, **opts):
        self._lib = capi.load()
        self.plan = plan
        self.bounded = bounded
        self.opts = recon_opts(**opts)
        h = C.c_void_p()
        if bounded:
            capi.check(self._lib.lct_recon_create_bounded(plan.handle, C.byref(self.opts),
                                                          int(piece_views), C.byref(h)),
                       "lct_recon_create_bounded")
        else:
            capi.check(self._lib.lct_recon_create(plan.handle, C.byref(self.opts), C.byref(h)),
                       "lct_recon_create")
        self._h = h
        first, count = C.c_int64(), C.c_int64()
        capi.check(self._lib.lct_recon_fan_range(h, C.byref(first), C.byref(count)))
        self.fan_first, self.fan_count = first.value, count.value
        info = plan.info
        self.image_shape = (info.n_blocks_run * BLOCK_SLICES, info.ig.ny, info.ig.nx)

    def run(self, fan, image=None, stream=None, fan_view0: int = 0):
        """fan: CUDA tensor or host tensor/array [views][nt][ns] float32 holding fan views from
        `fan_view0` on (all readings by default; at least [fan_first, fan_first+fan_count));
        host memory is copied inside, pinned is fastest.  image: same side as wanted, or None
        (a CUDA tensor is allocated)."""
        torch = _torch()
        if image is None:
            image = torch.empty(self.image_shape, dtype=torch.float32, device="cuda")
        g = self.plan.info.ctg
        _check_views(fan, self.fan_first, self.fan_count, int(fan_view0), g.ns * g.nt)
        if int(np.prod(image.shape)) < int(np.prod(self.image_shape)):
            raise ValueError(f"image smaller than {self.image_shape}")
        f_dev, f_ptr = _ptr(fan)
        i_dev, i_ptr = _ptr(image)
        s = stream if stream is not None else _stream()
        capi.check(self._lib.lct_recon_run(self._h, f_ptr, int(fan_view0), int(f_dev), i_ptr,
                                           int(i_dev), s), "lct_recon_run")
        return image

    def run_file(self, fan_path, image_path=None, image=None, stream=None):
        """lct_recon_run_file: the fan read from the reference's raw file (view v at byte
        (v + DataOffset) * nt * ns * 4), the volume written to image_path and/or the host array
        `image` (C-contiguous float32 of image_shape).  Returns `image`."""
        if image_path is None and image is None:
            raise ValueError("give image_path, image or both")
        ip = None
        if image is not None:
            on_dev, ip = _ptr(image)
            if on_dev:
                raise ValueError("run_file writes a host volume")
            if int(np.prod(image.shape)) < int(np.prod(self.image_shape)):
                raise ValueError(f"image smaller than {self.image_shape}")
        s = stream if stream is not None else _stream()
        capi.check(self._lib.lct_recon_run_file(
            self._h, str(fan_path).encode(), None if image_path is None else str(image_path).encode(),
            ip, s), "lct_recon_run_file")
        return image

    def device_bytes(self) -> int:
        n = C.c_int64()
        capi.check(self._lib.lct_recon_device_bytes(self._h, C.byref(n)))
        return n.value

    def stats(self) -> capi.ReconStats:
        st = capi.ReconStats()
        capi.check(self._lib.lct_recon_stats_get(self._h, C.byref(st)))
        return st

    def set_learned(self, cnn, bound: float | None = None) -> None:
        """Fuse the learned correction (learn.CNN, inference workspace of this image's ny x nx)
        after backprojection; None turns it off.  run() then returns the corrected volume."""
        if cnn is None:
            capi.check(self._lib.lct_recon_set_learned(self._h, None, 0.0), "lct_recon_set_learned")
            self._cnn = None
            return
        from .learn import DEFAULT_BOUND

        b = DEFAULT_BOUND if bound is None else bound
        capi.check(self._lib.lct_recon_set_learned(self._h, cnn._h, float(b)),
                   "lct_recon_set_learned")
        self._cnn = cnn  # keep it alive while fused

    def learned_info(self) -> dict:
        ms, rej = C.c_float(), C.c_int64()
        capi.check(self._lib.lct_recon_learned_info(self._h, C.byref(ms), C.byref(rej)))
        return {"ms": ms.value, "rejected": rej.value}

    def autotune(self) -> tuple[int, int]:
        nz, mb = C.c_int(), C.c_int()
        capi.check(self._lib.lct_recon_autotune(self._h, C.byref(nz), C.byref(mb)))
        return nz.value, mb.value

    def last_times(self) -> dict:
        t = (C.c_float * 5)()
        capi.check(self._lib.lct_recon_last_times(self._h, t))
        return dict(zip(["h2d", "rebin", "filter", "backproject", "d2h"], list(t)))

    def io_times(self) -> dict:
        """lct_recon_io_times: seconds of the last run_file -- reads (summed over the reader
        threads), pipeline waits for fan chunks, pipeline waits for writer slots."""
        t = (C.c_float * 3)()
        capi.check(self._lib.lct_recon_io_times(self._h, t))
        return dict(zip(["read", "wait_read", "wait_write"], list(t)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.lct_recon_destroy(h)
            self._h = None


class Batch:
    """lct_batch: many independent scans reconstructed together -- one CUDA-graph launch per
    stage, one persistent work-list backprojection over all scans' tiles."""

    def __init__(self, plans: list[Plan], **opts):
        self._lib = capi.load()
        self.plans = list(plans)
        self.opts = recon_opts(**opts)
        arr = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        h = C.c_void_p()
        capi.check(self._lib.lct_batch_create(arr, len(plans), C.byref(self.opts), C.byref(h)),
                   "lct_batch_create")
        self._h = h
        self.fan_ranges = []
        for i in range(len(plans)):
            f, c = C.c_int64(), C.c_int64()
            capi.check(self._lib.lct_batch_fan_range(h, i, C.byref(f), C.byref(c)))
            self.fan_ranges.append((f.value, c.value))
        self.image_shapes = [(p.info.n_blocks_run * BLOCK_SLICES, p.info.ig.ny, p.info.ig.nx)
                             for p in plans]

    def run(self, fans, images=None, fan_view0=None, stream=None):
        torch = _torch()
        n = len(self.plans)
        if images is None:
            images = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in self.image_shapes]
        for i, (f, p) in enumerate(zip(fans, self.plans)):
            first, count = self.fan_ranges[i]
            g = p.info.ctg
            _check_views(f, first, count, int((fan_view0 or [0] * n)[i]), g.ns * g.nt,
                         what=f"fan {i}")
        for i, sh in zip(images, self.image_shapes):
            if int(np.prod(i.shape)) < int(np.prod(sh)):
                raise ValueError(f"image smaller than {sh}")
        fp = [_ptr(f) for f in fans]
        ip = [_ptr(i) for i in images]
        if len({d for d, _ in fp}) != 1 or len({d for d, _ in ip}) != 1:
            raise ValueError("all fans (and all images) must be on the same side")
        v0 = (C.c_int64 * n)(*(fan_view0 or [0] * n))
        fa = (C.c_void_p * n)(*[p for _, p in fp])
        ia = (C.c_void_p * n)(*[p for _, p in ip])
        s = stream if stream is not None else _stream()
        capi.check(self._lib.lct_batch_run(self._h, fa, v0, int(fp[0][0]), ia, int(ip[0][0]), s),
                   "lct_batch_run")
        return images

    def stats(self) -> capi.ReconStats:
        st = capi.ReconStats()
        capi.check(self._lib.lct_batch_stats_get(self._h, C.byref(st)))
        return st

    def last_times(self) -> dict:
        t = (C.c_float * 5)()
        capi.check(self._lib.lct_batch_last_times(self._h, t))
        return dict(zip(["upload", "rebin", "filter", "backproject", "download"], list(t)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.lct_batch_destroy(h)
            self._h = None


def _check_views(x, first: int, count: int, view0: int, plane: int, what: str = "fan") -> None:
    """The buffer must hold views [first, first + count) counted from view0 (the C ABI takes a
    bare pointer and cannot check it)."""
    if first < view0:
        raise ValueError(f"{what} starts at view {view0} but the run needs view {first}")
    need = (first + count - view0) * plane
    have = int(np.prod(x.shape)) if hasattr(x, "shape") else None
    if have is not None and have < need:
        raise ValueError(f"{what} holds {have // plane} views from view {view0}; the run reads "
                         f"views {first}..{first + count - 1}")


def _ptr(x):
    """(on_device, pointer) of a torch tensor or numpy array (C-contiguous float32)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        if x.dtype != torch.float32 or not x.is_contiguous():
            raise ValueError("expected a contiguous float32 tensor")
        return x.is_cuda, x.data_ptr()
    a = np.asarray(x)
    if a.dtype != np.float32 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float32 array")
    return False, a.ctypes.data


# ------------------------------------------------------------------------------------------
# mirror of the reference's data model
# ------------------------------------------------------------------------------------------
class GPUMemoryCtrl:
    """Include/GPUMemoryCtrl.h:6-62: one allocation at a time; allocate_memory refuses a second
    one and returns False; copies check the size.  Backed by a torch CUDA tensor."""

    def __init__(self, dtype=np.float32):
        self.s = 0
        self._t = None
        self._dtype = dtype

    def allocate_memory(self, ele_num: int = 1) -> bool:
        if self.s != 0:
            return False
        torch = _torch()
        try:
            self._t = torch.empty(int(ele_num), dtype=torch.float32, device="cuda")
        except RuntimeError:
            return False
        self.s = int(ele_num)
        return True

    def free_memory(self) -> bool:
        self._t = None
        self.s = 0
        return True

    def copy_from_CPU(self, src: np.ndarray, ele_num: int, offset: int = 0) -> bool:
        if self.s - offset < ele_num:
            return False
        torch = _torch()
        self._t[offset:offset + ele_num].copy_(torch.from_numpy(np.ascontiguousarray(src).reshape(-1)[:ele_num]))
        return True

    def copy_to_CPU(self, dst: np.ndarray, ele_num: int, offset: int = 0) -> bool:
        if self.s - offset < ele_num:
            return False
        dst.reshape(-1)[:ele_num] = self._t[offset:offset + ele_num].cpu().numpy()
        return True

    def get_pointer(self, offset: int = 0) -> int:
        return self._t.data_ptr() + 4 * offset

    @property
    def tensor(self):
        return self._t


class CTDataCPU:
    def __init__(self, tube_angles, table_positions, size_proj, size_rebin, size_image):
        self.proj = np.zeros(size_proj, dtype=np.float32)
        self.rebin = np.zeros(size_rebin, dtype=np.float32)
        self.image = np.zeros(size_image, dtype=np.float32)
        self.tube_angles = np.array(tube_angles, dtype=np.float32)
        self.table_positions = np.array(table_positions, dtype=np.float32)

    def proj_(self): return self.proj
    def rebin_(self): return self.rebin
    def image_(self): return self.image
    def tube_angles_(self): return self.tube_angles
    def table_positions_(self): return self.table_positions


class CTDataGPU:
    """Include/DataStructs.h:213-229 (+ the device fan block the product rebins from)."""

    def __init__(self):
        self.ctg_gpu = None
        self.ig_gpu = None
        self.proj_gpu = GPUMemoryCtrl()
        self.img_gpu = GPUMemoryCtrl()
        self.betas_gpu = GPUMemoryCtrl()
        self.fan_gpu = GPUMemoryCtrl()


class BlockInfoCursor:
    """BlockInfo (Include/DataStructs.h:281-311): the current block; update() advances."""

    def __init__(self, blocks):
        self._blocks = blocks
        self._i = 0

    def update(self, ri=None, ctg=None, ig=None, data_cpu=None):
        self._i += 1

    def _cur(self):
        return self._blocks[min(self._i, len(self._blocks) - 1)]

    def block_idx(self): return self._i
    def block_proj_start(self): return self._cur().block_proj_start
    def block_proj_end(self): return self._cur().block_proj_end
    def block_start(self): return self._cur().block_start
    def block_end(self): return self._cur().block_end
    def block_slice_start(self): return self._cur().block_slice_start
    def block_slice_end(self): return self._cur().block_slice_end


class ReconData:
    """ReconData(fp): reads ViewAngleFile / CouchPosFile after ViewOffset and plans the blocks
    (Src/DataStructs.cpp:121-250).  Missing files raise ParameterError (the reference calls
    exit(1), :132-135)."""

    def __init__(self, fp: FileParams):
        d = Path(fp.RawDataDir)
        raw = Path(fp.RawDataDir + fp.DataInterpFile)
        if not raw.is_file():
            raise ParameterError("Raw data file not found.")
        n = fp.Readings + fp.ViewOffset
        ang = _read_f32(Path(fp.RawDataDir + fp.ViewAngleFile), n)[fp.ViewOffset:]
        pos = _read_f32(Path(fp.RawDataDir + fp.CouchPosFile), n)[fp.ViewOffset:]
        p = capi.ScanParams()
        p.ns, p.nt, p.ds, p.dt, p.pitch_value = fp.Ns, fp.Nt, fp.Ds, fp.Dt, fp.PitchValue
        p.nx, p.ny, p.dx, p.dz = fp.Nx, fp.Ny, fp.Dx, fp.Dz
        p.offset_x, p.offset_y = fp.OffsetX, fp.OffsetY
        p.readings, p.view_offset, p.data_offset = fp.Readings, fp.ViewOffset, fp.DataOffset
        p.r_src_to_iso, p.central_channel, p.n_proj_turn = fp.RSrcToIso, fp.CentralChannel, fp.NProjTurn
        p.max_blocks = fp.MaxBlocks
        self.fp = fp
        self.plan = Plan(params=p, angles32=ang, zpos32=pos)
        info = self.plan.info
        self.ctg = info.ctg
        self.ig = info.ig
        self.ri = info
        self.fi = (fp.RawDataDir, fp.DataInterpFile, fp.OutputDir, fp.OutputName)
        ns, nt = self.ctg.ns, self.ctg.nt
        self.data_cpu = CTDataCPU(ang, pos, ns * nt * self.ctg.n_angle_add, ns * nt * self.ctg.n_angle,
                                  info.ig.nx * info.ig.ny * info.n_blocks_run * BLOCK_SLICES)
        self.data_gpu = CTDataGPU()
        self.data_gpu.betas_gpu.allocate_memory(fp.Readings)
        self.bi = BlockInfoCursor(self.plan.blocks)

    def ctg_(self): return self.ctg
    def ig_(self): return self.ig
    def ri_(self): return self.ri
    def bi_(self): return self.bi
    def data_cpu_(self): return self.data_cpu
    def data_gpu_(self): return self.data_gpu

    def n_blocks(self) -> int:
        """Blocks FDKReconstructor runs (n_blocks, capped by the optional MaxBlocks key)."""
        return self.ri.n_blocks_run


def _read_f32(path: Path, n: int) -> np.ndarray:
    if not path.is_file():
        raise ParameterError("Raw data file not found.")
    a = np.fromfile(path, dtype=np.float32, count=n)
    if a.size < n:
        raise ParameterError(f"{path} holds {a.size} floats, {n} needed")
    return a


# ------------------------------------------------------------------------------------------
# stages
# ------------------------------------------------------------------------------------------
class _Bound:
    """Addressing of a stage's legacy texture binding: LCT_ADDR_LEGACY reproduces attributes
    captured at bind time (Clamp on the first bind, Border afterwards)."""

    def __init__(self, addr: int):
        self.addr = addr
        self.binds = 0

    def next_addr(self) -> int:
        self.binds += 1
        if self.addr == capi.ADDR_LEGACY:
            return capi.ADDR_CLAMP if self.binds == 1 else capi.ADDR_BORDER
        return self.addr


class Rebiner:
    def __init__(self, interp: int = capi.INTERP_TEX8, addr: int = capi.ADDR_BORDER):
        self.interp = interp
        self._bind = _Bound(addr)

    def rebin(self, mr: ReconData) -> None:
        raise NotImplementedError

    def _upload(self, mr: ReconData):
        g = mr.ctg
        dg = mr.data_gpu
        n = g.ns * g.nt * g.n_angle_add
        if dg.fan_gpu.s != n:
            dg.fan_gpu.free_memory()
            dg.fan_gpu.allocate_memory(n)
        dg.fan_gpu.copy_from_CPU(mr.data_cpu.proj, n)
        # CUDA/Rebiner.cu:142 -- the rebinner allocates projGpu (refused if still allocated)
        dg.proj_gpu.allocate_memory(g.ns * g.nt * g.n_angle)

    def _call(self, fn, mr: ReconData, *args):
        self._upload(mr)
        g = mr.ctg
        dg = mr.data_gpu
        capi.check(fn(C.byref(g), dg.fan_gpu.get_pointer(), dg.proj_gpu.get_pointer(), *args,
                      _stream()), fn.__name__)


class NullRebinerGPU(Rebiner):
    def rebin(self, mr):
        self._call(capi.lib().lct_rebin_null, mr, self._bind.next_addr())


class HelicalConeBeamFan2ParRebinerGPU(Rebiner):
    def rebin(self, mr):
        self._call(capi.lib().lct_rebin_fan2par, mr, self.interp, self._bind.next_addr())


class PiOriRebiner(Rebiner):
    def rebin(self, mr):
        self._call(capi.lib().lct_rebin_pi_ori, mr, self.interp, self._bind.next_addr())


class PreWeighting:
    def weighting(self, mr: ReconData) -> int:
        raise NotImplementedError


class NULLPreWeighting(PreWeighting):
    def weighting(self, mr):
        return 1


class PiOriPreWeighting(PreWeighting):
    def weighting(self, mr):
        st = capi.lib().lct_weight_pi_ori(C.byref(mr.ctg), mr.data_gpu.proj_gpu.get_pointer(), _stream())
        if st != capi.LCT_OK:
            return -1
        try:
            _torch().cuda.current_stream().synchronize()
        except RuntimeError:
            return -1
        return 1


class Filter:
    """Filter::filter (CUDA/Filter.cu:52-73): taps from the calculate_filter hook, convolution
    in place on projGpu, then the filtered block is copied to host `rebin`."""

    def __init__(self, mode: int = capi.FILTER_FP32, copy_to_host: bool = True):
        self.mode = mode
        self.copy_to_host = copy_to_host

    def calculate_filter(self, h: np.ndarray, ctg) -> None:
        raise NotImplementedError

    def filter(self, mr: ReconData) -> None:
        torch = _torch()
        g = mr.ctg
        h = np.zeros(2 * g.ns, dtype=np.float32)
        self.calculate_filter(h, g)
        d_h = torch.from_numpy(h).cuda()
        lib = capi.lib()
        capi.check(lib.lct_filter_rows(g.ns, d_h.data_ptr(), mr.data_gpu.proj_gpu.get_pointer(),
                                       g.n_angle * g.nt, self.mode, _stream()), "lct_filter_rows")
        if self.copy_to_host:
            mr.data_gpu.proj_gpu.copy_to_CPU(mr.data_cpu.rebin, g.ns * g.nt * g.n_angle)


class RampFilterGPU(Filter):
    def calculate_filter(self, h, ctg):
        capi.check(capi.lib().lct_filter_taps(capi.FILTER_RAMLAK, capi.WINDOW_NONE, ctg.ns, ctg.ds,
                                              h.ctypes.data))


class WindowedFilterGPU(Filter):
    """New: a Shepp-Logan or windowed ramp (the reference's SmoothWindow header is empty)."""

    def __init__(self, kind=capi.FILTER_SHEPP_LOGAN, window=capi.WINDOW_NONE, **kw):
        super().__init__(**kw)
        self.kind, self.window = kind, window

    def calculate_filter(self, h, ctg):
        capi.check(capi.lib().lct_filter_taps(self.kind, self.window, ctg.ns, ctg.ds, h.ctypes.data))


class Backprojector:
    def __init__(self, interp: int = capi.INTERP_TEX8, addr: int = capi.ADDR_BORDER):
        self.interp = interp
        self._bind = _Bound(addr)

    def backproject(self, mr: ReconData) -> None:
        raise NotImplementedError

    def _run(self, fn, mr: ReconData):
        g, ig = mr.ctg, mr.ig
        dg = mr.data_gpu
        addr = self._bind.next_addr()
        bps = mr.bi.block_proj_start()
        # CUDA/Backprojector.cu:145 -- betas of the block's rebinned views
        dg.betas_gpu.copy_from_CPU(mr.data_cpu.tube_angles[bps + g.add_projections:], g.n_angle)
        dg.img_gpu.allocate_memory(ig.nx * ig.ny * ig.nz)
        capi.check(fn(C.byref(g), C.byref(ig), dg.betas_gpu.get_pointer(), dg.proj_gpu.get_pointer(),
                      dg.img_gpu.get_pointer(), self.interp, addr, _stream()), fn.__name__)
        # CUDA/Backprojector.cu:138 -- the backprojector frees projGpu
        n = ig.nx * ig.ny * ig.nz
        dg.img_gpu.copy_to_CPU(mr.data_cpu.image[n * mr.bi.block_idx():], n)
        dg.proj_gpu.free_memory()
        dg.img_gpu.free_memory()


class HelicalConeBeamFanRebinBackprojectorGPU(Backprojector):
    def backproject(self, mr):
        self._run(capi.lib().lct_backproject_par, mr)


class PiOriBackprojectorGPU(Backprojector):
    def backproject(self, mr):
        self._run(capi.lib().lct_backproject_pi_ori, mr)


class RawDataReader:
    """Src/DataReader.cpp:8-19 with 64-bit offsets; a short read raises (the reference leaves
    stale data)."""

    def readData(self, mr: ReconData) -> None:
        g = mr.ctg
        path = mr.fp.RawDataDir + mr.fp.DataInterpFile
        n = g.ns * g.nt * g.n_angle_add
        off = (mr.bi.block_proj_start() + mr.fp.DataOffset) * g.ns * g.nt * 4
        if off < 0:
            raise ParameterError("block view window starts before the raw file")
        with open(path, "rb") as f:
            f.seek(off)
            a = np.frombuffer(f.read(4 * n), dtype=np.float32)
        if a.size < n:
            raise ParameterError("raw file shorter than the block view window")
        mr.data_cpu.proj[:] = a


class RawImageWriter:
    """Src/ImageWriter.cpp:9-43: the volume as raw float32 [z][y][x], and rebin.raw."""

    def writeImage(self, mr: ReconData) -> None:
        out = Path(mr.fp.OutputDir)
        out.mkdir(parents=True, exist_ok=True)
        mr.data_cpu.image.tofile(out / mr.fp.OutputName)
        mr.data_cpu.rebin.tofile(out / "rebin.raw")


class Reconstructor:
    def reconstruct(self, mr: ReconData) -> None:
        raise NotImplementedError


class FDKReconstructor(Reconstructor):
    """Src/Reconstructor.cpp:11-49: per block read -> rebin -> weighting -> filter ->
    backproject -> BlockInfo::update."""

    def __init__(self, rbn: Rebiner, flt: Filter, bp: Backprojector, pw: PreWeighting):
        self.rbn, self.flt, self.bp, self.pw = rbn, flt, bp, pw
        self.dr = RawDataReader()

    def reconstruct(self, mr: ReconData) -> None:
        for _ in range(mr.n_blocks()):
            self.dr.readData(mr)
            self.rbn.rebin(mr)
            if self.pw.weighting(mr) != 1:
                raise capi.LctError(capi.LCT_ERR_CUDA, "weighting")
            self.flt.filter(mr)
            self.bp.backproject(mr)
            mr.bi.update(mr.ri, mr.ctg, mr.ig, mr.data_cpu)


class ReconstrctorAbstractFactory:
    """Src/ReconstructorAbstractFactory.cpp:11-33.  `if (str.find("fdk"))` is true for every
    name in which "fdk" does not start at index 0 (npos is non-zero), so the reference builds
    the helical FDK pipeline for those and fails (exit(1)) only for names starting with "fdk";
    this keeps that rule and raises ValueError instead of exiting."""

    def createReconstructor(self, name: str, *, interp=capi.INTERP_TEX8, addr=capi.ADDR_BORDER,
                            filter_mode=capi.FILTER_FP32) -> Reconstructor:
        if name.find("fdk") != 0:
            return FDKReconstructor(HelicalConeBeamFan2ParRebinerGPU(interp, addr),
                                    RampFilterGPU(filter_mode),
                                    HelicalConeBeamFanRebinBackprojectorGPU(interp, addr),
                                    NULLPreWeighting())
        raise ValueError("Error happens when building reconstructor.")
