"""Filter taps: Ram-Lak bit-exact with the reference's own RampFilterGPU::calculate_filter
(tests/golden/taps.json), the closed forms of Shepp-Logan and the windows against numerical
integration of h(n) = (1/ds) 2 int_0^1/2 f W(f) cos(2 pi n f) df."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from listctrecons_b200 import capi

TAPS = json.loads((Path(__file__).resolve().parent / "golden" / "taps.json").read_text())


def _taps(kind, window, ns, ds):
    h = np.zeros(2 * ns, dtype=np.float32)
    capi.check(capi.load().lct_filter_taps(kind, window, ns, ds, h.ctypes.data))
    return h


@pytest.mark.parametrize("rec", TAPS, ids=[f"ns{r['ns']}" for r in TAPS])
def test_ramlak_bit_exact_with_reference(rec):
    ref = np.array(rec["h"], dtype=np.float32)
    got = _taps(capi.FILTER_RAMLAK, capi.WINDOW_NONE, rec["ns"], rec["ds"])
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    # the oracle's restatement too
    assert np.array_equal(orc.ramp_taps(rec["ns"], rec["ds"]).view(np.uint32), ref.view(np.uint32))


def test_ramlak_known_values():
    ds = 0.6
    h = _taps(capi.FILTER_RAMLAK, capi.WINDOW_NONE, 64, ds).astype(np.float64)
    n = np.arange(-64, 64)
    assert h[64] == pytest.approx(1 / (4 * ds), rel=1e-7)
    even = (n % 2 == 0) & (n != 0)
    assert np.all(np.abs(h[even]) < 1e-12)
    odd = n % 2 == 1
    np.testing.assert_allclose(h[odd], -1.0 / (n[odd] ** 2 * math.pi ** 2 * ds), rtol=1e-6)


def _numeric(window, kind, n, ds, m=20001):
    f = np.linspace(0.0, 0.5, m)
    W = np.ones_like(f)
    if kind == capi.FILTER_SHEPP_LOGAN:
        W = W * np.sinc(f)
    if window == capi.WINDOW_HANN:
        W = W * (0.5 + 0.5 * np.cos(2 * np.pi * f))
    elif window == capi.WINDOW_HAMMING:
        W = W * (0.54 + 0.46 * np.cos(2 * np.pi * f))
    elif window == capi.WINDOW_COSINE:
        W = W * np.cos(np.pi * f)
    y = f * W * np.cos(2 * np.pi * n * f)
    return 2.0 * np.trapezoid(y, f) / ds


@pytest.mark.parametrize("kind", [capi.FILTER_RAMLAK, capi.FILTER_SHEPP_LOGAN])
@pytest.mark.parametrize("window", [capi.WINDOW_NONE, capi.WINDOW_HANN, capi.WINDOW_HAMMING, capi.WINDOW_COSINE])
def test_windowed_taps_match_integral(kind, window):
    ns, ds = 32, 0.8
    h = _taps(kind, window, ns, ds).astype(np.float64)
    for n in [0, 1, 2, 3, 7, 12]:
        assert h[ns + n] == pytest.approx(_numeric(window, kind, n, ds), abs=2e-6)
        assert h[ns - n] == pytest.approx(h[ns + n], rel=1e-6, abs=1e-9)


def test_shepp_logan_closed_form():
    ds = 0.6
    h = _taps(capi.FILTER_SHEPP_LOGAN, capi.WINDOW_NONE, 50, ds).astype(np.float64)
    n = np.arange(-50, 50)
    np.testing.assert_allclose(h, -2.0 / (math.pi ** 2 * ds * (4 * n.astype(float) ** 2 - 1)), rtol=1e-6)
