"""Known-answer tests of the CPU oracle (derived from the reference's formulas)."""
import math

import numpy as np
import pytest

import oracle as orc


def _geom(**kw):
    g = orc.Geom()
    base = dict(orbit=2 * math.pi / 100, orbit_start=0.0, ns=16, nt=4, ws=7.5, wt=1.5,
                n_angle=20, n_angle_add=40, ds=1.0, dt=1.0, pitch=4.0, source_z0=-2.0, dso=570.0,
                n_proj_turn=100, z_dir=1, add_projections=10)
    base.update(kw)
    for k, v in base.items():
        setattr(g, k, v)
    return g


def test_rebin_integer_shift_is_a_copy():
    # ds chosen so alpha(is)/orbit is an exact integer for every column: weights vanish
    g = _geom(ns=5, ws=2.0)
    g.orbit = 0.25
    g.ds = g.dso * g.orbit  # alpha/orbit = is - ws
    rng = np.random.default_rng(0)
    fan = rng.standard_normal((g.n_angle_add, g.nt, g.ns)).astype(np.float32)
    for interp in (orc.EXACT, orc.TEXEMU):
        out = orc.rebin_fan2par(g, fan, interp=interp)
        for ia in range(g.n_angle):
            for is_ in range(g.ns):
                np.testing.assert_array_equal(out[ia, :, is_], fan[ia + 10 + is_ - 2, :, is_])


def test_null_rebin_is_offset_copy():
    g = _geom()
    fan = np.arange(g.n_angle_add * g.nt * g.ns, dtype=np.float32).reshape(g.n_angle_add, g.nt, g.ns)
    np.testing.assert_array_equal(orc.rebin_null(g, fan), fan[10:30])


def test_texemu_weights_are_8bit():
    g = _geom(ns=64, ws=31.5)
    idx, w = orc.rebin_fan2par_index(g, orc.TEXEMU)
    assert np.all(np.abs(w * 256 - np.round(w * 256)) < 1e-6)
    idx_e, w_e = orc.rebin_fan2par_index(g, orc.EXACT)
    assert np.max(np.abs((idx + w) - (idx_e + w_e))) <= 0.5 / 256 + 1e-6


def test_filter_delta_row_returns_taps():
    ns = 32
    h = orc.ramp_taps(ns, 1.0)
    row = np.zeros((1, ns), dtype=np.float32)
    row[0, 5] = 1.0
    out = orc.filter_rows(h, row)
    # out[is] = h[is - 5 + ns]
    np.testing.assert_array_equal(out[0], h[np.arange(ns) - 5 + ns].astype(np.float64))
    seq = orc.filter_rows(h, row, mode=1)
    np.testing.assert_array_equal(seq[0], out[0])


def test_backprojection_of_constant_is_normalised():
    # constant filtered data c inside the detector: every pair contributes c*(ww+ww2)=c, so each
    # voxel gets c * 2*pi (the 2*pi/(a_max-a_min) scale of a full window)
    g = _geom(ns=200, ws=99.5, nt=64, wt=31.5, n_angle=300, n_angle_add=320, pitch=10.0,
              source_z0=-5.0, n_proj_turn=100, dt=1.0, ds=1.0)
    ig = orc.Img()
    ig.nx, ig.ny, ig.nz, ig.wx, ig.wy, ig.wz, ig.dx, ig.dy, ig.dz = 8, 8, 4, 3.5, 3.5, 0.0, 2.0, 2.0, 0.5
    proj = np.full((g.n_angle, g.nt, g.ns), 3.0, dtype=np.float32)
    betas = (np.arange(g.n_angle) * g.orbit).astype(np.float32)
    img = orc.bp_par(g, ig, betas, proj, interp=orc.EXACT)
    np.testing.assert_allclose(img, 3.0 * 2 * math.pi, rtol=1e-6)


def test_simulator_line_integral_of_centered_sphere():
    # a sphere of radius r at the isocentre: the central ray crosses 2r
    e = np.zeros((1, 16))
    e[0, 3:6] = 20.0
    e[0, 6:15] = np.eye(3).reshape(-1)
    e[0, 15] = 0.02
    ns, nt = 9, 3
    out = orc.sim_project(e, ns, nt, 1.0, 1.0, 4.0, 1.0, 570.0, np.array([0.3]), np.array([0.0]),
                          0, 1, 0.0, 1)
    assert out[0, 1, 4] == pytest.approx(0.02 * 40.0, rel=1e-6)
    # a ray at fan angle a passes R sin a from the centre
    a = 3 * 1.0 / 570.0
    d = 570.0 * math.sin(a)
    assert out[0, 1, 7] == pytest.approx(0.02 * 2 * math.sqrt(400 - d * d), rel=1e-5)


def test_poisson_noise_statistics():
    e = np.zeros((1, 16))
    e[0, 3:6] = 100.0
    e[0, 6:15] = np.eye(3).reshape(-1)
    e[0, 15] = 0.01
    ns, nt = 1, 4000
    ang = np.zeros(1)
    zs = np.zeros(1)
    clean = orc.sim_project(e, ns, nt, 1.0, 1e-4, 0.0, (nt - 1) / 2, 570.0, ang, zs, 0, 1, 0.0, 3)
    noisy = orc.sim_project(e, ns, nt, 1.0, 1e-4, 0.0, (nt - 1) / 2, 570.0, ang, zs, 0, 1, 1e5, 3)
    p = float(clean.mean())
    lam = 1e5 * math.exp(-p)
    counts = 1e5 * np.exp(-noisy.astype(np.float64))
    assert counts.mean() == pytest.approx(lam, rel=3e-3)
    assert counts.var() == pytest.approx(lam, rel=0.1)


@pytest.mark.parametrize("interp", [orc.EXACT, orc.TEXEMU])
@pytest.mark.parametrize("addr", [orc.BORDER, orc.CLAMP])
def test_column_order_backprojection_is_bit_identical(interp, addr):
    # partial windows at both ends (n_angle below a turn plus the slab's reach), a conjugate
    # that steps back by half a turn, offsets off the voxel grid, a negative couch direction
    g = _geom(ns=40, ws=19.25, nt=8, wt=3.5, n_angle=150, n_angle_add=170, pitch=6.0,
              source_z0=-3.0, n_proj_turn=100, dt=1.1, ds=1.3, z_dir=-1)
    ig = orc.Img()
    ig.nx, ig.ny, ig.nz, ig.wx, ig.wy, ig.wz, ig.dx, ig.dy, ig.dz = 12, 10, 32, 5.8, 4.3, 0.0, 1.7, 1.7, 0.31
    rng = np.random.default_rng(5)
    proj = rng.standard_normal((g.n_angle, g.nt, g.ns)).astype(np.float32)
    betas = np.mod(0.3 + np.arange(g.n_angle) * g.orbit, 2 * math.pi).astype(np.float32)
    a = orc.bp_par(g, ig, betas, proj, interp=interp, addr=addr)
    b = orc.bp_par_cols(g, ig, betas, proj, interp=interp, addr=addr)
    np.testing.assert_array_equal(a, b)
    c = orc.bp_par_cols(g, ig, betas, proj, interp=interp, addr=addr, rows=(3, 7))
    np.testing.assert_array_equal(c[:, 3:7], a[:, 3:7])
    d = orc.bp_par_cols(g, ig, betas, proj, interp=interp, addr=addr, ystep=3)
    np.testing.assert_array_equal(d[:, ::3], a[:, ::3])
    assert not d[:, 1::3].any()


def test_matrix_filter_matches_direct_sums():
    ns = 48
    rng = np.random.default_rng(2)
    rows = rng.standard_normal((7, ns)).astype(np.float32)
    for h in (orc.ramp_taps(ns, 0.6), orc.shepp_logan_taps(ns, 0.6)):
        a = orc.filter_rows(h, rows)
        b = orc.filter_rows_fp64(h, rows)
        np.testing.assert_allclose(b, a, rtol=0, atol=1e-13 * np.abs(a).max())
