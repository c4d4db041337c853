"""Bounded device memory and runs straight from the reference's raw files.

A bounded recon keeps fan, filtered and quad views in rings and the volume in a four-slab ring;
a scan of six blocks with small pieces makes every ring wrap several times.  Each view is still
uploaded, rebinned and filtered once by the same kernels, so the volume must equal the unbounded
device-resident run's bit for bit -- from a host fan, a device fan, and from the raw file through
the reader and writer threads (lct_recon_run_file), into pinned, pageable and device volumes --
while the device footprint stays below the unbounded recon's.  A short or missing file is an LCT_ERR_IO, not a partial volume."""
import numpy as np
import pytest

from listctrecons_b200 import capi
from listctrecons_b200.recon import Plan, Reconstruction
from listctrecons_b200.scan import Phantom, simulate_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scan6(small_geo, cuda):
    geo = small_geo.with_blocks(6)
    p = Plan(geo)
    assert p.info.n_blocks_run == 6
    lo = min(p.blocks[0].block_start, p.blocks[5].block_end)
    hi = max(p.blocks[0].block_start, p.blocks[5].block_end)
    ph = Phantom.random(8, seed=21, fov_radius=14.0, z_lo=lo, z_hi=hi, semi=(2.0, 9.0))
    fan = simulate_gpu(geo, ph, i0=1e5, seed=4)
    return dict(geo=geo, plan=p, fan=fan)


OPTS = [
    dict(interp=capi.INTERP_EXACT, filter_mode=capi.FILTER_BF16X6, addr=capi.ADDR_BORDER),
    dict(interp=capi.INTERP_TEX8, filter_mode=capi.FILTER_FP32, addr=capi.ADDR_CLAMP),
]


@pytest.mark.parametrize("opts", OPTS, ids=["exact-bf16x6-border", "tex8-fp32-clamp"])
def test_bounded_runs_are_bit_identical(scan6, opts):
    import torch

    p, fan = scan6["plan"], scan6["fan"]
    ref_r = Reconstruction(p, mode=capi.MODE_SCAN, **opts)
    ref = ref_r.run(fan).cpu().numpy()
    b = Reconstruction(p, bounded=True, piece_views=24, mode=capi.MODE_SCAN, **opts)
    assert b.device_bytes() < ref_r.device_bytes()
    # host fan -> host volume (fan ring + volume ring)
    h_fan = fan.cpu().pin_memory()
    h_img = torch.empty(b.image_shape, dtype=torch.float32).pin_memory()
    b.run(h_fan, h_img)
    np.testing.assert_array_equal(h_img.numpy(), ref)
    # device fan -> device volume (read and written in place)
    d_img = torch.full(b.image_shape, float("nan"), dtype=torch.float32, device="cuda")
    b.run(fan, d_img)
    np.testing.assert_array_equal(d_img.cpu().numpy(), ref)
    # again, over the rings' previous contents
    h_img.fill_(float("nan"))
    b.run(h_fan, h_img)
    np.testing.assert_array_equal(h_img.numpy(), ref)
    # pageable volume: slabs copied out of the pinned slots by the writer threads
    p_img = np.full(b.image_shape, np.nan, dtype=np.float32)
    b.run(h_fan, p_img)
    np.testing.assert_array_equal(p_img, ref)


def test_unbounded_streamed_run_into_pageable_volume(scan6):
    """A host fan streams; a pageable volume is downloaded once after the pipeline."""
    p, fan = scan6["plan"], scan6["fan"]
    opts = OPTS[0]
    r = Reconstruction(p, mode=capi.MODE_SCAN, **opts)
    ref = r.run(fan).cpu().numpy()
    p_img = np.full(r.image_shape, np.nan, dtype=np.float32)
    r.run(fan.cpu().pin_memory(), p_img)
    np.testing.assert_array_equal(p_img, ref)


@pytest.mark.parametrize("bounded", [True, False])
def test_run_file_reads_and_writes_the_reference_files(scan6, tmp_path, bounded):
    from listctrecons_b200.scan import write_scan_files

    p, fan = scan6["plan"], scan6["fan"]
    opts = OPTS[0]
    ref = Reconstruction(p, mode=capi.MODE_SCAN, **opts).run(fan).cpu().numpy()
    write_scan_files(scan6["geo"], fan.cpu().numpy(), tmp_path / "data", tmp_path / "out")
    r = Reconstruction(p, bounded=bounded, piece_views=24 if bounded else 0, mode=capi.MODE_SCAN,
                       **opts)
    out = tmp_path / "out" / "volume.raw"
    img = np.full(r.image_shape, np.nan, dtype=np.float32)
    r.run_file(tmp_path / "data" / "proj.raw", image_path=out, image=img)
    np.testing.assert_array_equal(img, ref)
    io = r.io_times()  # the readers read something; waits are never negative
    assert io["read"] > 0.0 and io["wait_read"] >= 0.0 and io["wait_write"] >= 0.0
    np.testing.assert_array_equal(np.fromfile(out, dtype=np.float32).reshape(ref.shape), ref)
    # pageable volume only (the writer threads copy it, no file)
    img.fill(np.nan)
    r.run_file(tmp_path / "data" / "proj.raw", image=img)
    np.testing.assert_array_equal(img, ref)
    # file only, twice (the pinned staging is reused)
    out2 = tmp_path / "out" / "volume2.raw"
    for _ in range(2):
        r.run_file(tmp_path / "data" / "proj.raw", image_path=out2)
        np.testing.assert_array_equal(np.fromfile(out2, dtype=np.float32).reshape(ref.shape), ref)


def test_run_file_refuses_short_and_missing_files(scan6, tmp_path):
    p, fan = scan6["plan"], scan6["fan"]
    r = Reconstruction(p, bounded=True, piece_views=24, mode=capi.MODE_SCAN,
                       interp=capi.INTERP_EXACT)
    short = tmp_path / "short.raw"
    f = fan.cpu().numpy()
    f[: r.fan_first + r.fan_count - 1].tofile(short)  # one view short of the run's last
    img = np.zeros(r.image_shape, dtype=np.float32)
    with pytest.raises(capi.LctError) as e:
        r.run_file(short, image=img)
    assert e.value.status == capi.LCT_ERR_IO
    with pytest.raises(capi.LctError) as e:
        r.run_file(tmp_path / "missing.raw", image=img)
    assert e.value.status == capi.LCT_ERR_IO
