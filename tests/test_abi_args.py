"""Argument checks of the C ABI that need no GPU: every entry point below rejects a missing
handle, a null buffer, a non-positive size or an out-of-range option with LCT_ERR_ARG before it
touches the device."""
import ctypes as C

import numpy as np

from listctrecons_b200 import capi


def test_cnn_entry_points_reject_bad_arguments():
    lib = capi.load()
    n = C.c_int64()
    assert lib.lct_cnn_param_count(C.byref(n)) == capi.LCT_OK and n.value == 57249
    assert lib.lct_cnn_param_count(None) == capi.LCT_ERR_ARG
    h = C.c_void_p()
    for args in [(0, 8, 8, 0, 0), (4, 0, 8, 0, 0), (4, 8, -1, 0, 0), (4, 8, 8, 2, 0),
                 (4, 8, 1 << 30, 0, 0)]:
        assert lib.lct_cnn_create(*args, C.byref(h)) == capi.LCT_ERR_ARG, args
    assert lib.lct_cnn_create(4, 8, 8, 0, 0, None) == capi.LCT_ERR_ARG
    buf = np.zeros(16, np.float32)
    p = buf.ctypes.data
    assert lib.lct_cnn_set_params(None, p, 0) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_get_params(None, p, 0) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_get_grads(None, p, 0) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_set_scales(None, 1.0, 1.0) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_forward(None, p, 1, None, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_backward(None, p, p, 1, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_adam_step(None, 1e-3, 0.9, 0.999, 1e-8, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_train_step(None, p, p, 1, 1e-3, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_infer_volume(None, p, p, 1, 0.1, None, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_last_loss(None, None) == capi.LCT_ERR_ARG
    assert lib.lct_cnn_get_shape(None, None, None, None) == capi.LCT_ERR_ARG
    lib.lct_cnn_destroy(None)  # a no-op


def test_recon_learned_and_batch_reject_bad_arguments():
    lib = capi.load()
    assert lib.lct_recon_set_learned(None, None, 0.1) == capi.LCT_ERR_ARG
    assert lib.lct_recon_learned_info(None, None, None) == capi.LCT_ERR_ARG
    h = C.c_void_p()
    assert lib.lct_batch_create(None, 0, None, C.byref(h)) == capi.LCT_ERR_ARG
    assert lib.lct_batch_run(None, None, None, 0, None, 0, None) == capi.LCT_ERR_ARG


def test_simulator_and_voxeliser_reject_bad_arguments():
    lib = capi.load()
    buf = np.zeros(64, np.float64)
    p = buf.ctypes.data
    # voxeliser: null, too many ellipsoids, non-positive sizes, sub-sampling out of range
    assert lib.lct_voxelise(None, 1, 4, 4, 4, 0, 0, 0, 1, 1, 1, 2, p, None) == capi.LCT_ERR_ARG
    assert lib.lct_voxelise(p, 129, 4, 4, 4, 0, 0, 0, 1, 1, 1, 2, p, None) == capi.LCT_ERR_ARG
    assert lib.lct_voxelise(p, 1, 0, 4, 4, 0, 0, 0, 1, 1, 1, 2, p, None) == capi.LCT_ERR_ARG
    assert lib.lct_voxelise(p, 1, 4, 4, 4, 0, 0, 0, 1, 1, 1, 0, p, None) == capi.LCT_ERR_ARG
    assert lib.lct_voxelise(p, 1, 4, 4, 4, 0, 0, 0, 1, 1, 1, 17, p, None) == capi.LCT_ERR_ARG
    # simulator: reversed view range, non-positive spacing
    assert lib.lct_sim_project(p, 1, 8, 2, 1.0, 1.0, 3.5, 0.5, 570.0, p, p, 5, 4, 1e5, 1, p,
                               None) == capi.LCT_ERR_ARG
    assert lib.lct_sim_project(p, 1, 8, 2, 0.0, 1.0, 3.5, 0.5, 570.0, p, p, 0, 4, 1e5, 1, p,
                               None) == capi.LCT_ERR_ARG


def test_bounded_and_file_runs_reject_bad_arguments():
    lib = capi.load()
    h = C.c_void_p()
    assert lib.lct_recon_create_bounded(None, None, 0, C.byref(h)) == capi.LCT_ERR_ARG
    assert lib.lct_recon_create_bounded(None, None, -1, C.byref(h)) == capi.LCT_ERR_ARG
    n = C.c_int64()
    assert lib.lct_recon_device_bytes(None, C.byref(n)) == capi.LCT_ERR_ARG
    assert lib.lct_recon_run_file(None, b"x", b"y", None, None) == capi.LCT_ERR_ARG
