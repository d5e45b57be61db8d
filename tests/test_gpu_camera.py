"""Thin-lens camera and pixel filters (box, triangle, gaussian, mitchell, sinc)
against the oracle at matched seeds, and the three schedules on them."""
import numpy as np
import pytest

import oracle
from vision_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {
    'triangle': dict(filter={'type': 'triangle', 'param': {'radius': [1.0, 1.0]}}),
    'gaussian': dict(filter={'type': 'gaussian', 'param': {'radius': [1.5, 1.5], 'sigma': 0.5}}),
    'mitchell': dict(filter={'type': 'mitchell', 'param': {'radius': [2.0, 2.0]}}),
    'sinc': dict(filter={'type': 'sinc', 'param': {'radius': [2.0, 2.0], 'tau': 3.0}}),
    'thin_lens': dict(lens={'lens_radius': 0.04, 'focal_distance': 1.6}),
    'thin_lens_gaussian': dict(lens={'lens_radius': 0.02, 'focal_distance': 1.2},
                               filter={'type': 'gaussian', 'param': {'radius': [1.0, 1.5], 'sigma': 0.6}}),
}


def _scene(case, width=48, height=48):
    sc = scenes.box_room(width=width, height=height)
    cam = sc['camera']
    spec = CASES[case]
    if 'filter' in spec:
        cam['param']['filter'] = spec['filter']
    if 'lens' in spec:
        cam['type'] = 'thin_lens'
        cam['param'].update(spec['lens'])
    return sc


@pytest.mark.parametrize('case', sorted(CASES))
def test_camera_matched_seed_parity(vb, gpu_ctx, case):
    # Same sampler streams on both sides; the filter offset, its weight and
    # the lens sample feed the same paths, so per-pixel agreement holds for
    # almost every pixel (FP32 transcendental / FMA differences flip a rare
    # decision) and the film means agree.
    s = vb.Scene(gpu_ctx, _scene(case)).build_accel()
    o = oracle.OracleScene(s)
    s.render(0, 8)
    g = s.film()
    c = o.render(0, 8)
    assert np.all(np.isfinite(g))
    diff = np.abs(g[..., :3] - c[..., :3])
    close = diff <= 1e-3 * (1.0 + np.abs(c[..., :3]))
    assert close.all(-1).mean() >= 0.97, close.all(-1).mean()
    assert abs(g[..., :3].mean() - c[..., :3].mean()) < 2e-3 * c[..., :3].mean()


@pytest.mark.parametrize('case', ['mitchell', 'thin_lens_gaussian'])
def test_camera_schedules_give_the_same_film(vb, gpu_ctx, case):
    # The filter weight rides with the path (wavefront: the radiance
    # record's w), so all three schedules still write identical films.
    films = {}
    for schedule in ('grid', 'persistent', 'wavefront'):
        s = vb.Scene(gpu_ctx, _scene(case, 37, 29)).build_accel()
        s.set_schedule(schedule)
        s.render(0, 6, fp64=True)
        films[schedule] = (s.film(), s.film(vb.FILM_SUM64))
    for schedule in ('persistent', 'wavefront'):
        assert np.array_equal(films['grid'][0], films[schedule][0]), schedule
        assert np.array_equal(films['grid'][1], films[schedule][1]), schedule


def test_filtered_films_converge_to_the_box_film(vb, gpu_ctx):
    # A normalised filter only reweights where within the footprint a
    # pixel's samples land: over the flat-lit back wall the films agree with
    # the box film, and the lens blur leaves the mean unchanged.
    means = {}
    for case in ('box', 'gaussian', 'thin_lens'):
        sc = scenes.box_room(width=32, height=32) if case == 'box' else _scene(case, 32, 32)
        s = vb.Scene(gpu_ctx, sc).build_accel()
        s.render(0, 256)
        means[case] = s.film()[..., :3].mean()
    for case in ('gaussian', 'thin_lens'):
        assert abs(means[case] - means['box']) < 0.02 * means['box'], (case, means)
