"""The film's pictures (exposure, tone mappers, sRGB gamma, 8-bit output)
against a numpy restatement of the reference's output path:
output = tm(1 - exp(-L * exposure)) (normal.cpp:86-101), final picture =
srgb(tm(output)) or tm(output) for HDR files (postprocessor.cpp:13-22,
pipeline.cpp:313-329)."""
import numpy as np
import pytest

from vision_b200 import scenes

pytestmark = pytest.mark.gpu


def _tm(x, kind):
    x = x.astype(np.float32)
    if kind == 'aces':
        return np.clip((x * (np.float32(2.51) * x + np.float32(0.03))) /
                       (x * (np.float32(2.43) * x + np.float32(0.59)) + np.float32(0.14)), 0, 1)
    if kind == 'reinhard':
        return x / (x + np.float32(1))
    return x


def _srgb(v):
    v = v.astype(np.float64)
    return np.where(v <= 0.0031308, 12.92 * v, 1.055 * np.power(np.maximum(v, 0), 1 / 2.4) - 0.055)


@pytest.mark.parametrize('kind', ['linear', 'aces', 'reinhard'])
def test_pictures_follow_the_output_path(vb, gpu_ctx, kind):
    sc = scenes.box_room(width=40, height=30)
    rc = sc['camera']['param']['radiance_collector']['param']
    rc['exposure'] = 1.7
    rc['tone_mapper'] = {'type': kind}
    s = vb.Scene(gpu_ctx, sc).build_accel()
    s.render(0, 4)
    lin = s.film()[..., :3]
    out = _tm(1.0 - np.exp(-lin * np.float32(1.7)), kind)
    np.testing.assert_allclose(s.film(vb.FILM_EXPOSED)[..., :3], out, atol=2e-6, rtol=1e-5)
    final = _tm(out, kind)
    np.testing.assert_allclose(s.film(vb.FILM_HDR)[..., :3], final, atol=2e-6, rtol=1e-5)
    disp = _srgb(final)
    np.testing.assert_allclose(s.film(vb.FILM_DISPLAY)[..., :3], disp, atol=1e-5, rtol=1e-5)
    rgba = s.film(vb.FILM_RGBA8)
    q = np.rint(np.clip(disp, 0, 1) * 255.0)
    assert np.abs(rgba[..., :3].astype(np.int32) - q).max() <= 1
    assert (rgba[..., :3] == q).mean() > 0.99
    assert np.all(rgba[..., 3] == 255)
    for which in (vb.FILM_EXPOSED, vb.FILM_HDR, vb.FILM_DISPLAY):
        assert np.all(s.film(which)[..., 3] == 1.0)


def test_full_hd_picture(vb, gpu_ctx):
    # A 1920 x 1080 film (one frame, depth 2): the picture kernels at the
    # size a display pipeline reads, against the same restatement.
    sc = scenes.box_room(width=1920, height=1080, max_depth=2)
    sc['camera']['param']['radiance_collector']['param']['tone_mapper'] = {'type': 'aces'}
    s = vb.Scene(gpu_ctx, sc).build_accel()
    s.render(0, 1)
    lin = s.film()[..., :3]
    disp = _srgb(_tm(_tm(1.0 - np.exp(-lin), 'aces'), 'aces'))
    np.testing.assert_allclose(s.film(vb.FILM_DISPLAY)[..., :3], disp, atol=1e-5, rtol=1e-5)
    rgba = s.film(vb.FILM_RGBA8)
    assert np.abs(rgba[..., :3].astype(np.int32) - np.rint(np.clip(disp, 0, 1) * 255.0)).max() <= 1
