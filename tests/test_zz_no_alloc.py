"""lct_backproject_par_noalloc -- backprojection for callers that cannot let the library
allocate device memory (their host budgets all device memory, or an allocation must never stall
or fail mid-acquisition).  Its scratch is a fixed 64 MiB array compiled into the library.

Checked through the C ABI against the allocating entry point lct_backproject_par, on two calls
in a row with different data (the shared array keeps the previous call's contents), in both
interpolation modes, on a block that takes the quad path (the one that uses the array); and an
oversize block is refused before anything runs.  This file is collected last so a run that stops
at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan

pytestmark = pytest.mark.gpu


def _quad_path(g, ig) -> bool:
    out = C.c_int(-1)
    capi.check(capi.load().lct_backproject_par_quad_path(C.byref(g), C.byref(ig), C.byref(out)))
    return out.value == 1


def _run(fn, g, ig, betas, proj, interp):
    import torch

    img = torch.full((ig.nz, ig.ny, ig.nx), float("nan"), dtype=torch.float32, device="cuda")
    capi.check(fn(C.byref(g), C.byref(ig), betas.data_ptr(), proj.data_ptr(), img.data_ptr(),
                  interp, capi.ADDR_BORDER, torch.cuda.current_stream().cuda_stream), fn.__name__)
    torch.cuda.synchronize()
    return img.cpu().numpy()


@pytest.mark.parametrize("interp", [capi.INTERP_EXACT, capi.INTERP_TEX8])
def test_noalloc_matches_allocating_entry_point(small_geo, cuda, interp):
    import torch

    lib = capi.load()
    p = Plan(small_geo)
    g, ig = p.info.ctg, p.info.ig
    assert _quad_path(g, ig)  # the block uses the shared scratch array
    b0 = p.blocks[0].block_proj_start + g.add_projections
    betas = torch.from_numpy(np.ascontiguousarray(p.angles32[b0:b0 + g.n_angle])).cuda()
    rng = np.random.default_rng(123)
    for call in range(2):  # second call: different data over the same shared scratch
        proj = torch.from_numpy(rng.standard_normal((g.n_angle, g.nt, g.ns)).astype(np.float32)).cuda()
        ref = _run(lib.lct_backproject_par, g, ig, betas, proj, interp)
        got = _run(lib.lct_backproject_par_noalloc, g, ig, betas, proj, interp)
        assert np.isfinite(got).all()
        err = orc.rel_l2(got, ref)
        assert err < 1e-5, (call, err)


def test_noalloc_refuses_blocks_beyond_its_scratch(cuda):
    import torch

    from listctrecons_b200.scan import ScanGeometry

    geo = ScanGeometry(ns=736, nt=64, ds=0.6, dt=0.6, npt=1152, pitch=0.8, nx=64, ny=64, dx=0.5,
                       dz=0.5, readings=11520)
    p = Plan(geo)
    g, ig = p.info.ctg, p.info.ig
    need = g.n_angle * (g.nt + 3) * (g.ns + 3) * 16
    assert need > 64 << 20
    # the refusal happens on the quad path; checked on the host before anything is called
    assert ig.nz <= 32 and _quad_path(g, ig)
    # buffers at their full sizes, so even a call that went on to launch would stay in bounds
    proj = torch.zeros(g.n_angle * g.nt * g.ns, dtype=torch.float32, device="cuda")
    betas = torch.zeros(g.n_angle, dtype=torch.float32, device="cuda")
    img = torch.full((ig.nz * ig.ny * ig.nx,), 7.0, dtype=torch.float32, device="cuda")
    st = capi.load().lct_backproject_par_noalloc(C.byref(g), C.byref(ig), betas.data_ptr(),
                                                 proj.data_ptr(), img.data_ptr(),
                                                 capi.INTERP_EXACT, capi.ADDR_BORDER, None)
    assert st == capi.LCT_ERR_SCRATCH
    assert b"scratch" in capi.load().lct_status_string(st)
    torch.cuda.synchronize()
    assert (img.cpu().numpy() == 7.0).all()  # nothing was launched
