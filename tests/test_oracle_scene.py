"""The oracle's own scene ingestion (oracle/scene.py, restated from the
reference's shapes, materials, lights, warpers and sensor without the
library) against the flat scene the library exports: the same triangles,
records and sampling tables, so a scene-layer mistake on either side fails
here instead of being shared by both sides of the parity tests."""
import numpy as np
import pytest

from oracle import scene as oscene
from vision_b200 import scenes

# Arrays computed in the same FP32 order on both sides agree to rounding;
# the procedural sky is evaluated in FP64 by the oracle and FP32 by the
# library (texels within 1 %, sampling distributions within 2 %).
ENV_TOL = {'env_tex': 1e-2, 'env_marginal_func': 1e-3, 'env_cond_func': 1e-2}
ALIAS_KEYS = ('prim_alias', 'light_alias', 'env_marginal', 'env_cond')


def _alias_rows(arr, key, info):
    if key == 'env_cond':
        w = int(arr['env']['width'][0])
        return arr[key].reshape(-1, w)
    if key == 'prim_alias':
        rows = []
        for L in arr['lights']:
            if L['shape'] == 0:
                rows.append(arr[key][L['alias_offset']:L['alias_offset'] + L['prim_count']])
        return rows
    return [arr[key]]


def _compare(vb, ctx, sc):
    mine, info = oscene.build(sc)
    s = vb.Scene(ctx, sc).build_accel()
    lib = {k: (s.export(k).view(a.dtype) if a.dtype.names else s.export(k, a.dtype)) for k, a in mine.items()}
    assert info['prim_count'] == s.info()['prim_count']
    for k, a in mine.items():
        e = lib[k]
        assert a.shape == e.shape, k
        if k in ALIAS_KEYS:
            ra, re_ = _alias_rows(mine, k, info), _alias_rows(lib, k, info)
            tol = 2e-2 if k.startswith('env') else 1e-3
            for x, y in zip(ra, re_):
                da, de = oscene.alias_distribution(x), oscene.alias_distribution(y)
                assert np.all(np.abs(da - de) <= 1e-7 + tol * de), k
            continue
        for f in (a.dtype.names or [None]):
            x, y = (a[f], e[f]) if f else (a, e)
            if np.issubdtype(x.dtype, np.floating):
                fin = np.isfinite(y)
                assert np.array_equal(np.isfinite(x), fin), (k, f)
                tol = ENV_TOL.get(k, 2e-5 if k != 'env' else 1e-4)
                np.testing.assert_allclose(x[fin], y[fin], rtol=tol, atol=1e-6, err_msg='%s.%s' % (k, f))
            else:
                assert np.array_equal(x, y), (k, f)


@pytest.mark.parametrize('name', ['box_room', 'box_room_rgb_light', 'material_room', 'substrate_room',
                                  'plastic_room', 'point_lights', 'srgb', 'many_lights', 'large_scene_small',
                                  'sphere_trs', 'principled_room', 'mix_room', 'metallic_room'])
def test_oracle_scene_equals_library_export(vb, host_ctx, name):
    if name == 'box_room':
        sc = scenes.box_room(64, 48, sampler='pcg')
    elif name == 'box_room_rgb_light':
        sc = scenes.box_room(32, 32, rgb_light=True)
    elif name == 'material_room':
        sc = scenes.material_room(32, 32)
    elif name == 'substrate_room':
        sc = scenes.substrate_room(32, 32)
    elif name == 'plastic_room':
        sc = scenes.plastic_room(32, 32)
    elif name == 'principled_room':
        sc = scenes.principled_room(32, 32)
    elif name == 'mix_room':
        sc = scenes.mix_room(32, 32)
    elif name == 'metallic_room':
        sc = scenes.metallic_room(32, 32)
    elif name == 'point_lights':
        sc = scenes.point_light_room(32, 32, light_sampler='power')
    elif name == 'srgb':
        sc = scenes.material_room(32, 32)
        sc.pop('spectrum')
    elif name == 'many_lights':
        sc = scenes.many_lights(64, 64, emitters=500, integrator='pt', dimension=4)
    elif name == 'large_scene_small':
        sc = scenes.large_scene(width=40, height=40, subdivisions=4, grid=60, tiles=4, sky_width=256,
                                sky_height=128)
    else:
        sc = scenes.box_room(32, 32)
        sc['shapes'].append({'type': 'sphere', 'name': 'ball', 'param': {
            'radius': 0.08, 'sub_div': 16, 'material': 'ShortBox',
            'transform': {'type': 'trs', 'param': {'t': [0.17, 0.38, 0.12], 'r': [0, 1, 0, 30],
                                                   's': [1.0, 1.5, 1.0]}}}})
    _compare(vb, host_ctx, sc)


def test_oracle_scene_of_the_benchmark(vb, host_ctx):
    # The 2,327,680-triangle large scene and its 2048 x 1024 sky.
    _compare(vb, host_ctx, scenes.large_scene())


def test_oracle_scene_unsupported_is_reported():
    sc = scenes.box_room(16, 16)
    sc['materials'][0]['type'] = 'subsurface'
    with pytest.raises(oscene.Unsupported):
        oscene.build(sc)
