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
def test_wavefront_cache_frame_matches_one_kernel_frame(vb, gpu_ctx, room):
    # The wavefront frame (prefix passes through path_shade, query kernel,
    # compacted training suffixes) against the one-kernel frame k_cache_paths,
    # which restates the bounce loop separately: same sampler draws and
    # summation order, so almost every path is identical; a path through
    # several specular events can take another branch on a last-bit
    # difference.  One frame with the seeded initial weights (training happens
    # after the frame).
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
        q = s.cache_buffer('query_records')
        t = s.cache_buffer('train_records')
        out[schedule] = dict(valid=q['l_valid'][..., 3] != 0, qf=s.cache_buffer('query_features'),
                             rec=np.concatenate([q['t'], q['l_valid']], -1), tf=s.cache_buffer('train_features'),
                             bf=s.cache_buffer('suffix_features'), tg=s.cache_buffer('targets'),
                             sv=t['suffix_valid'], film=s.film())
    a, b = out['grid'], out['wavefront']
    assert (a['valid'] == b['valid']).mean() >= 0.995
    both = a['valid'] & b['valid']
    assert both.mean() > 0.3

    # Features are BF16 codes (compared exactly); records and targets are
    # FP32 sums whose last bits depend on how each kernel's multiply-adds were
    # contracted (compared to 1e-4 relative).
    def rows_equal(x, y):
        return np.all(x == y, axis=-1).mean()

    def rows_close(x, y):
        return np.all(np.abs(x - y) <= 1e-6 + 1e-4 * np.abs(x), axis=-1).mean()
    assert rows_equal(a['qf'][both], b['qf'][both]) >= 0.99
    assert rows_close(a['rec'][both], b['rec'][both]) >= 0.99
    for k in ('tf', 'bf'):
        assert rows_equal(a[k], b[k]) >= 0.98, k
    for k in ('tg', 'sv'):
        assert rows_close(a[k], b[k]) >= 0.98, k
    close = np.abs(a['film'] - b['film']) <= 1e-4 + 1e-3 * np.abs(a['film'])
    assert close.all(-1).mean() >= 0.99
    assert abs(a['film'][..., :3].mean() - b['film'][..., :3].mean()) <= 1e-3 * a['film'][..., :3].mean()
