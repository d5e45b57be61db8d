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


@pytest.mark.parametrize('room', ['box', 'materials'])
def test_wavefront_cache_frame_equals_megakernel(vb, gpu_ctx, room):
    # The wavefront frame (prefix passes, query kernel, compacted training
    # suffixes) makes the same draws and sums as the one-kernel frame: the
    # features, records, targets and film of a frame are identical.  One frame
    # with the seeded initial weights (training happens after the frame).
    if room == 'box':
        sc = scenes.box_room(80, 60, max_depth=8, dimension=3, sampler='pcg')
    else:
        sc = scenes.material_room(64, 48, dimension=3, sampler='pcg')
    out = {}
    for schedule in ('grid', 'wavefront'):
        s = vb.Scene(gpu_ctx, sc).build_accel()
        s.set_schedule(schedule)
        cache = vb.RadianceCache(gpu_ctx, seed=1)
        s.render_cached(cache, 0, 1, train_samples=700)
        bufs = {k: s.cache_buffer(k) for k in ('query_features', 'query_output', 'train_features', 'suffix_features',
                                               'suffix_output', 'targets')}
        q = s.cache_buffer('query_records')
        bufs['valid'] = q['l_valid'][..., 3]
        bufs['query_t'] = np.where(bufs['valid'][..., None] != 0, q['t'], 0)
        bufs['film'] = s.film()
        t = s.cache_buffer('train_records')
        bufs['suffix'] = t['suffix_valid']
        out[schedule] = bufs
    for k in out['grid']:
        assert np.array_equal(out['grid'][k], out['wavefront'][k]), k
    assert out['grid']['valid'].mean() > 0.3
