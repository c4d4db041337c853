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
