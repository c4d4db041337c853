"""Toeplitz-GEMM filter on tcgen05 against the FP64 oracle and the FP32 path.

BF16x3 (2-way bf16 splits, 3 products): rel-L2 <= 2e-4 on filtered rows -- the ramp filter's
cancellation amplifies the ~2^-16 product error -- and <= 1e-4 on reconstructed volumes.
BF16x6 (3-way splits, 6 products): rel-L2 <= 1e-5 on rows (FP32-level).  The device status
word stays clear (no bounded wait ran out)."""
import ctypes as C

import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi

pytestmark = pytest.mark.gpu


def _filter(rows, h, mode):
    import torch

    d_rows = torch.from_numpy(np.ascontiguousarray(rows)).cuda()
    d_h = torch.from_numpy(np.ascontiguousarray(h)).cuda()
    capi.check(capi.load().lct_filter_rows(rows.shape[-1], d_h.data_ptr(), d_rows.data_ptr(),
                                           rows.shape[0], mode, None), "lct_filter_rows")
    torch.cuda.synchronize()
    return d_rows.cpu().numpy()


@pytest.mark.parametrize("mode,tol", [(capi.FILTER_BF16X3, 2e-4), (capi.FILTER_BF16X6, 1e-5)])
@pytest.mark.parametrize("ns,nrows", [(96, 37), (101, 300), (736, 1000), (896, 129)])
def test_tc_filter_matches_oracle(cuda, ns, nrows, mode, tol):
    rng = np.random.default_rng(ns + nrows)
    # smooth rows plus noise, like rebinned line integrals
    x = np.linspace(0, 6, ns)
    rows = (2 + np.sin(x[None, :] * rng.uniform(0.5, 2, (nrows, 1))) +
            0.05 * rng.standard_normal((nrows, ns))).astype(np.float32)
    h = orc.shepp_logan_taps(ns, 0.6)
    got = _filter(rows, h, mode)
    ref = orc.filter_rows(h, rows, mode=0)
    fp32 = _filter(rows, h, capi.FILTER_FP32)
    err, err32 = orc.rel_l2(got, ref), orc.rel_l2(fp32, ref)
    print(f"ns={ns} rows={nrows} mode={mode}: tc rel_l2={err:.3e} fp32 rel_l2={err32:.3e}")
    assert err < tol
    code = C.c_int(-1)
    assert capi.load().lct_device_status(C.byref(code)) == capi.LCT_OK and code.value == 0


@pytest.mark.parametrize("mode", [capi.FILTER_BF16X3, capi.FILTER_BF16X6])
def test_tc_filter_volume(small_geo, cuda, mode):
    """Whole reconstruction with the tensor-core filter against the FP32-filter one."""
    import torch

    from listctrecons_b200.recon import Plan, Reconstruction
    from listctrecons_b200.scan import Phantom, simulate_gpu

    p = Plan(small_geo)
    ph = Phantom.random(6, seed=3, fov_radius=14.0, z_lo=p.blocks[0].block_start,
                        z_hi=p.blocks[-1].block_end, semi=(2.0, 9.0))
    fan = simulate_gpu(small_geo, ph, i0=1e5, seed=9)
    ref = Reconstruction(p, interp=capi.INTERP_EXACT).run(fan).cpu().numpy()
    for m in (capi.MODE_SCAN, capi.MODE_BLOCK):
        got = Reconstruction(p, interp=capi.INTERP_EXACT, filter_mode=mode, mode=m).run(fan)
        err = orc.rel_l2(got.cpu().numpy(), ref)
        print(f"volume mode={m} filter={mode}: rel_l2 vs FP32 filter = {err:.3e}")
        assert err < 1e-4
