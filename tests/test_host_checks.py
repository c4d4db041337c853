"""Host-side argument checks of the Python wrappers (no GPU): a fan buffer must hold the views a
run reads, counted from fan_view0, because the C ABI receives a bare pointer."""
import numpy as np
import pytest

from listctrecons_b200.recon import _check_views


def test_fan_view_range_check():
    plane = 4 * 8
    x = np.zeros((10, 4, 8), np.float32)
    _check_views(x, 5, 5, 0, plane)            # views 5..9 of a buffer starting at view 0
    _check_views(x[:5], 5, 5, 5, plane)        # the same views in a buffer starting at view 5
    with pytest.raises(ValueError):
        _check_views(x, 5, 6, 0, plane)        # view 10 is past the end
    with pytest.raises(ValueError):
        _check_views(x, 5, 5, 6, plane)        # buffer starts after the first needed view
    with pytest.raises(ValueError):
        _check_views(x[:5], 5, 5, 0, plane)    # a partial buffer passed with fan_view0 = 0


def test_reference_pi_window_bound(small_geo):
    """The reference's PI-window backprojector walks forward to a_min + n_proj_turn / 2 with no
    bound against n_angle (CUDA/Backprojector.cu:225).  The bench and the drop-in test run the
    reference's PI configuration only when a_middle + n_proj_turn / 2 stays below n_angle for every
    slice (a_min <= a_middle), so its betas reads stay inside the array: true for the test scan,
    false once the block holds too few views."""
    import ctypes as C
    from types import SimpleNamespace

    import bench
    from listctrecons_b200.recon import Plan

    p = Plan(small_geo)
    assert bench.pi_window_in_bounds(p)
    g = p.info.ctg
    short = type(g)()
    C.pointer(short)[0] = g  # a copy of the geometry with fewer views in the block
    short.n_angle = g.n_proj_turn // 2 + 1
    assert not bench.pi_window_in_bounds(SimpleNamespace(info=SimpleNamespace(ctg=short, ig=p.info.ig)))
