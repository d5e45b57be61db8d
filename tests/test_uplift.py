"""Accuracy of the RGB -> spectrum uplift table (reference
RGBToSpectrumTable::decode_albedo, src/render_core/spectra/hero.cpp:92-175).

The reference's coefficient table (srgb2spec.h) is a missing blob; the
library regenerates it with the published Jakob & Hanika (2019) fit.  This
checks the table the renderer uses by the quantity the method optimises: a
colour decoded to sigmoid coefficients, taken as a reflectance spectrum
s(lambda) = 1/2 + x / (2 sqrt(1 + x^2)), x = (c0 lambda + c1) lambda + c2,
lit by D65 and projected with the CIE 1931 matching functions back to linear
sRGB must give the colour back, within the CIELAB distance the method reaches
(Jakob & Hanika report round trips below visible differences, Delta E << 1)."""
import numpy as np
import pytest

from oracle.scene import tables

M_XYZ_TO_RGB = np.array([[3.240479, -1.537150, -0.498535], [-0.969256, 1.875991, 0.041556],
                         [0.055648, -0.204043, 1.057311]])


def _reflectance_rgb(c):
    t = tables()
    lam = 360.0 + np.arange(471)
    X, Y, Z, D = (t[k].astype(np.float64) for k in ('VS_CIE_X', 'VS_CIE_Y', 'VS_CIE_Z', 'VS_CIE_D65'))
    x = (c[0] * lam + c[1]) * lam + c[2]
    s = 0.5 + x / (2.0 * np.sqrt(1.0 + x * x))
    xyz = np.array([np.sum(s * D * X), np.sum(s * D * Y), np.sum(s * D * Z)]) / np.sum(D * Y)
    return M_XYZ_TO_RGB @ xyz


def _lab(rgb):
    inv = np.linalg.inv(M_XYZ_TO_RGB)
    r = (inv @ rgb) / (inv @ np.ones(3))
    f = np.where(r > (6 / 29) ** 3, np.cbrt(r), r / (3 * (6 / 29) ** 2) + 4 / 29)
    return np.array([116 * f[1] - 16, 500 * (f[0] - f[1]), 200 * (f[1] - f[2])])


def test_uplift_round_trip_random_colours(vb, host_ctx):
    rng = np.random.default_rng(2019)
    cols = rng.random((300, 3)).astype(np.float32)
    de, err = [], []
    for rgb in cols:
        out = _reflectance_rgb(host_ctx.rgb_to_spectrum(rgb, 0))
        err.append(np.abs(out - rgb).max())
        de.append(np.linalg.norm(_lab(out) - _lab(rgb.astype(np.float64))))
    de, err = np.array(de), np.array(err)
    # Measured: Delta E76 max 0.13, median 0.02; RGB error max 1.1e-3.
    assert de.max() < 0.5, de.max()
    assert np.median(de) < 0.05, np.median(de)
    assert err.max() < 3e-3, err.max()


@pytest.mark.parametrize('rgb', [[0.63, 0.065, 0.05], [0.14, 0.45, 0.091], [0.725, 0.725, 0.725], [1, 0, 0],
                                 [0, 1, 0], [0, 0, 1], [0.9, 0.9, 0.1], [0.02, 0.02, 0.9], [0.5, 0.0, 0.5]])
def test_uplift_round_trip_scene_and_gamut_colours(vb, host_ctx, rgb):
    # The box room's wall colours, a grey (the exact analytic path), the
    # primaries and saturated secondaries at the gamut boundary.
    rgb = np.array(rgb, np.float32)
    c = host_ctx.rgb_to_spectrum(rgb, 0)
    out = _reflectance_rgb(c)
    # Measured: Delta E76 at most 0.25 (a saturated blue near the gamut
    # corner, where the trilinear interpolation is coarsest).
    assert np.linalg.norm(_lab(out) - _lab(rgb.astype(np.float64))) < 0.5
    assert abs(c[3] - (0.212671 * rgb[0] + 0.715160 * rgb[1] + 0.072169 * rgb[2])) < 1e-6
    if rgb[0] == rgb[1] == rgb[2]:
        assert c[0] == 0.0 and c[1] == 0.0


def test_unbound_decode_scales(vb, host_ctx):
    # decode_unbound (hero.cpp:135-141): coefficients of rgb / (2 max) and the
    # scale 2 max, so an emitter colour above one keeps its chromaticity.
    rgb = np.array([17.0, 8.5, 4.25], np.float32)
    c = host_ctx.rgb_to_spectrum(rgb, 1)
    assert abs(c[3] - 34.0) < 1e-5
    out = _reflectance_rgb(c) * c[3]
    np.testing.assert_allclose(out, rgb, rtol=3e-3)
