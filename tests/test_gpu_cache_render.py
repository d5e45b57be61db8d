"""Cache-terminated rendering: paths that stop after two bounces into the
radiance cache.  The trained cache must recover the light that the same
two-bounce paths miss without it (the gain of the network over the method
without it), measured against an FP64 plain reference with independent
samples."""
import numpy as np
import pytest

from vision_b200 import scenes

pytestmark = pytest.mark.gpu


def _relmse(img, ref, eps=1e-2):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + eps)))


def _bright_room(w, h, max_depth, seed=0):
    # Walls and boxes at albedo 0.9, so that light beyond the second bounce is
    # a large share of the image (about a third here; about a tenth in the
    # standard room).
    sc = scenes.box_room(w, h, max_depth=max_depth, dimension=3, sampler='pcg', seed=seed)
    for m in sc['materials']:
        if m['type'] == 'diffuse':
            m['param']['color'] = [0.9, 0.9, 0.9]
    return sc


def test_cache_recovers_missing_light(vb, gpu_ctx):
    w = h = 96
    ref_scene = vb.Scene(gpu_ctx, _bright_room(w, h, 32, seed=91)).build_accel()
    ref_scene.render(0, 2048, fp64=True)
    ref = ref_scene.film(vb.FILM_SUM64)[..., :3] / 2048
    # The method without the network: the same paths cut after two bounces.
    cut = vb.Scene(gpu_ctx, _bright_room(w, h, 2)).build_accel()
    cut.render(0, 128)
    img_cut = cut.film()[..., :3]
    sc = _bright_room(w, h, 32)
    train = vb.Scene(gpu_ctx, sc).build_accel()
    cached = vb.Scene(gpu_ctx, sc).build_accel()
    cache = vb.RadianceCache(gpu_ctx, seed=1)
    cache.set_optimizer(lr=3e-3)
    train.render_cached(cache, 0, 800, train_samples=w * h)
    cached.render_cached(cache, 0, 128, train_samples=0)
    img = cached.film()[..., :3]
    assert np.all(np.isfinite(img))
    missing = ref.mean() - img_cut.mean()
    assert missing > 0.2 * ref.mean(), (ref.mean(), img_cut.mean())
    # The cache restores most of the missing energy and lowers the error.
    assert abs(img.mean() - ref.mean()) < 0.25 * missing, (img.mean(), ref.mean(), img_cut.mean())
    assert _relmse(img, ref) < 0.5 * _relmse(img_cut, ref), (_relmse(img, ref), _relmse(img_cut, ref))


def test_cached_render_needs_three_wavelengths(vb, gpu_ctx):
    s = vb.Scene(gpu_ctx, scenes.box_room(16, 16, dimension=4)).build_accel()
    cache = vb.RadianceCache(gpu_ctx, seed=1)
    with pytest.raises(vb.UnsupportedError):
        s.render_cached(cache, 0, 1)
