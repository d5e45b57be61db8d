"""Scene-layer semantics of the C-ABI host side (no GPU)."""
import json
import math
import os

import numpy as np
import pytest

from vision_b200 import scenes

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_box_room_counts(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.box_room()).build_accel()
    i = s.info()
    assert i['prim_count'] == 5 * 2 + 2 * 12 + 2
    assert i['light_count'] == 1
    assert i['spectrum_dim'] == 4 and i['max_depth'] == 8
    assert (i['width'], i['height']) == (256, 256)


def test_quad_matches_reference_layout(vb, host_ctx):
    # Quad::init (quad.cpp:21-50): P = (w,0,h),(w,0,-h),(-w,0,h),(-w,0,-h); tris (0,1,2),(2,1,3).
    sc = scenes.box_room(width=4, height=4)
    s = vb.Scene(host_ctx, sc)
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    np.testing.assert_array_equal(pos[:4], [[0.5, 0, 0.5], [0.5, 0, -0.5], [-0.5, 0, 0.5], [-0.5, 0, -0.5]])
    np.testing.assert_array_equal(idx[:2], [[0, 1, 2], [2, 1, 3]])
    # Geometric normal of the floor points up (+y), into the room.
    p = pos[idx[0]]
    ng = np.cross(p[0] - p[2], p[1] - p[2])
    assert ng[1] > 0 and abs(ng[0]) < 1e-6 and abs(ng[2]) < 1e-6


def test_walls_face_into_the_room(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.box_room(width=4, height=4))
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    center = np.array([0, 0.5, 0], np.float32)
    for t in range(10):  # the five wall quads
        p = pos[idx[t]]
        ng = np.cross(p[0] - p[2], p[1] - p[2])
        assert np.dot(ng, center - p.mean(0)) > 0, t
    # The light quad faces down.
    p = pos[idx[-1]]
    assert np.cross(p[0] - p[2], p[1] - p[2])[1] < 0


def test_cube_matches_reference_sizes(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.box_room(width=4, height=4))
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    tall = pos[np.unique(idx[10:22])]
    assert abs(tall[:, 1].max() - 0.6) < 1e-5 and abs(tall[:, 1].min()) < 1e-5
    # Rotated 15 degrees about y: edge length along the rotated x axis stays 0.3.
    e = np.linalg.norm(tall[None] - tall[:, None], axis=-1)
    assert np.any(np.isclose(e, 0.3, atol=1e-5))


def test_camera_look_at(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.box_room(width=4, height=4))
    cam = s.export('camera', np.float32)
    c2w = cam[:16].reshape(4, 4)  # column-major: c2w[c][r]
    np.testing.assert_allclose(c2w[3, :3], [0, 0.5, 1.85], atol=1e-6)
    fwd = c2w[2, :3]
    np.testing.assert_allclose(fwd, [0, 0, -1], atol=1e-6)
    assert abs(cam[16] - math.tan(math.radians(20))) < 1e-6


@pytest.mark.parametrize('ftype, param, code, p0, p1', [
    ('box', {}, 0, 0.0, 0.0),
    ('triangle', {}, 1, 0.0, 0.0),
    ('gaussian', {}, 2, 1.0, 0.0),                  # GaussianFilter sigma default (gaussian.cpp:21)
    ('gaussian', {'sigma': 0.4}, 2, 0.4, 0.0),
    ('mitchell', {}, 3, 1.0 / 3.0, 1.0 / 3.0),      # b, c defaults (mitchell.cpp:20-21)
    ('sinc', {}, 4, 3.0, 0.0),                      # tau default (sinc.cpp:20)
])
def test_camera_filter_and_lens_parse(vb, host_ctx, ftype, param, code, p0, p1):
    sc = scenes.box_room(width=4, height=4)
    sc['camera']['type'] = 'thin_lens'
    sc['camera']['param'].update(lens_radius=0.05, focal_distance=2.5)
    sc['camera']['param']['filter'] = {'type': ftype, 'param': dict(param, radius=[1.25, 0.75])}
    cam = vb.Scene(host_ctx, sc).export('camera', np.float32)
    u = cam.view(np.uint32)
    assert cam.nbytes == 128
    np.testing.assert_allclose(cam[21:23], [1.25, 0.75])
    assert (u[26], u[27]) == (code, 1)
    np.testing.assert_allclose(cam[28:32], [0.05, 2.5, p0, p1], rtol=1e-6)


def test_unknown_filter_is_unsupported(vb, host_ctx):
    sc = scenes.box_room(width=4, height=4)
    sc['camera']['param']['filter'] = {'type': 'lanczos2', 'param': {}}
    with pytest.raises(vb.UnsupportedError):
        vb.Scene(host_ctx, sc)


def test_rgb_light_is_normalised(vb, host_ctx):
    # Light::Light + NumberArray::normalize: [17,17,17] -> colour 1, scale 17.
    s = vb.Scene(host_ctx, scenes.box_room(width=4, height=4, rgb_light=True))
    L = s.export('lights', np.float32).reshape(-1, 28)
    Lu = L.view(np.uint32)
    assert Lu[0, 5] == 0  # RGB emitter
    assert L[0, 6] == np.float32(17.0)
    np.testing.assert_array_equal(s.export('light_rgb', np.float32), [1, 1, 1])
    # decode_unbound of (1,1,1): grey -> c = 0, scale 2.
    np.testing.assert_array_equal(L[0, 8:12], [0, 0, 0, 2])


def test_alias_tables_match_reference_algorithm(vb, host_ctx):
    # An emissive inline mesh with uneven triangle areas; its per-primitive
    # alias table must equal the reference algorithm (golden restatement).
    rng = np.random.default_rng(3)
    n = 17
    P, I = [], []
    for t in range(n):
        base = rng.random(3) * 0.5
        a = 0.01 + 0.3 * rng.random()
        P += list(base) + list(base + [a, 0, 0]) + list(base + [0, 0, a])
        I += [3 * t, 3 * t + 2, 3 * t + 1]
    sc = scenes.box_room(width=4, height=4)
    sc['shapes'].append({'type': 'mesh', 'name': 'emitter', 'param': {
        'positions': P, 'indices': I, 'material': 'Light',
        'emission': {'type': 'area', 'param': {'color': [1, 1, 1], 'scale': 1.0}}}})
    s = vb.Scene(host_ctx, sc)
    L = s.export('lights', np.uint32).reshape(-1, 28)
    assert L.shape[0] == 2
    off, cnt = L[1, 3], L[1, 2]
    tab = s.export('prim_alias', np.uint8).view([('prob', np.float32), ('alias', np.uint32)])[off:off + cnt]
    pmf = s.export('prim_pmf', np.float32)[off:off + cnt]
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)[L[1, 1]:L[1, 1] + cnt]
    areas = []
    for t in idx:
        p = pos[t]
        areas.append(np.float32(0.5) * np.float32(np.linalg.norm(np.cross(p[0] - p[2], p[1] - p[2]).astype(np.float32))))
    # Reference Vose construction (alias.h:86-122), restated.
    w = [float(a) for a in areas]
    ratio = len(w) / sum(np.float64(x) for x in w)
    table = [[float(np.float32(x * ratio)), i] for i, x in enumerate(w)]
    over = [i for i, t in enumerate(table) if t[0] > 1.0]
    under = [i for i, t in enumerate(table) if not t[0] > 1.0]
    while over and under:
        o, u = over.pop(), under.pop()
        table[o][0] = float(np.float32(np.float32(table[o][0]) - (np.float32(1.0) - np.float32(table[u][0]))))
        table[u][1] = o
        if table[o][0] > 1.0:
            over.append(o)
        elif table[o][0] < 1.0:
            under.append(o)
    for i in over + under:
        table[i] = [1.0, i]
    np.testing.assert_allclose(tab['prob'], [t[0] for t in table], rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(tab['alias'], [t[1] for t in table])
    np.testing.assert_allclose(pmf, np.array(w) / np.sum(w), rtol=1e-5)


def test_golden_alias_tables(vb, host_ctx):
    for c in json.load(open(os.path.join(G, 'alias.json'))):
        # Build through the library with an emissive mesh whose triangle areas
        # are the golden weights.
        P, I = [], []
        for t, wgt in enumerate(c['weights']):
            a = math.sqrt(2.0 * wgt)
            P += [0, 0, 3 * t, a, 0, 3 * t, 0, 0, 3 * t + a]
            I += [3 * t, 3 * t + 2, 3 * t + 1]
        sc = scenes.box_room(width=4, height=4)
        sc['shapes'].append({'type': 'mesh', 'name': 'e', 'param': {
            'positions': P, 'indices': I, 'material': 'Light',
            'emission': {'type': 'area', 'param': {'color': [1, 1, 1]}}}})
        s = vb.Scene(host_ctx, sc)
        L = s.export('lights', np.uint32).reshape(-1, 28)
        off, cnt = L[1, 3], L[1, 2]
        pmf = s.export('prim_pmf', np.float32)[off:off + cnt]
        np.testing.assert_allclose(pmf, c['pmf'], rtol=1e-4)


def test_unsupported_light_in_light_sampler(vb, host_ctx):
    sc = scenes.box_room(width=4, height=4)
    sc['light_sampler']['param']['lights'] = [{'type': 'photometric', 'param': {}}]
    with pytest.raises(vb.UnsupportedError):
        vb.Scene(host_ctx, sc)


def test_environment_warper_matches_reference_construction(vb, host_ctx):
    # AliasTable2D::build (alias2d.cpp:30-66) from the weights of
    # SphericalMap::calculate_weights (spherical.cpp:187-213), restated here.
    sc = scenes.large_scene(width=8, height=8, subdivisions=1, grid=4, tiles=2, sky_width=64, sky_height=32)
    s = vb.Scene(host_ctx, sc)
    env = s.export('env', np.float32)
    W, H = env[32:34].view(np.uint32)
    tex = s.export('env_tex', np.float32).reshape(H, W, 4)
    idx = np.arange(W * H)
    theta = ((idx // H).astype(np.float32) + np.float32(0.5)) / np.float32(W)
    lum = (np.float32(0.212671) * tex[..., 0] + np.float32(0.715160) * tex[..., 1] +
           np.float32(0.072169) * tex[..., 2]).reshape(-1)
    w = (lum * np.sin(np.float32(np.pi) * theta).astype(np.float32)).astype(np.float32)
    cf = s.export('env_cond_func', np.float32)
    np.testing.assert_allclose(cf, w, rtol=2e-6, atol=1e-30)
    mf = s.export('env_marginal_func', np.float32)
    np.testing.assert_allclose(mf, w.reshape(H, W).astype(np.float64).sum(1) / W, rtol=1e-6)
    assert abs(env[35] - np.float32(mf.astype(np.float64).sum() / H)) <= 1e-6 * env[35]
    # The sky's sun lobe peaks near 5e4.
    assert 1.0e4 < tex[..., :3].max() <= 5.0e4 + 10


def test_large_scene_counts(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.large_scene(width=8, height=8, subdivisions=7, grid=1000, tiles=10,
                                              sky_width=64, sky_height=32))
    i = s.info()
    assert i['prim_count'] == 20 * 4 ** 7 + 2 * 1000 * 1000
    assert i['instance_count'] == 101
    types = s.export('materials', np.uint32).reshape(-1, 16)[:, 0]
    assert set(types.tolist()) == {2, 3, 4}


def test_bvh_collapse_setting(vb, host_ctx):
    # render_setting.bvh_collapse: "sah" (default: the SAH-optimal choice of
    # each wide node's children, fuller nodes) or "greedy";
    # render_setting.bvh_leaf_size: 1 to 3 triangles per leaf, or "auto"
    # (default: 1 for trees of 4096 primitives or more, else 3).
    counts = {}
    for collapse in ('greedy', 'sah'):
        for leaf in (1, 3):
            sc = scenes.large_scene(width=8, height=8, subdivisions=4, grid=100, tiles=2, sky_width=64, sky_height=32)
            sc['render_setting']['bvh_collapse'] = collapse
            sc['render_setting']['bvh_leaf_size'] = leaf
            s = vb.Scene(host_ctx, sc).build_accel()
            counts[collapse, leaf] = s.info()['bvh_node_count']
    assert counts['sah', 1] < counts['greedy', 1] and counts['sah', 3] < counts['greedy', 3]
    assert counts['sah', 3] < counts['sah', 1]
    sc = scenes.large_scene(width=8, height=8, subdivisions=4, grid=100, tiles=2, sky_width=64, sky_height=32)
    assert vb.Scene(host_ctx, sc).build_accel().info()['bvh_node_count'] == counts['sah', 1]
    small = {}
    for leaf in ('auto', 3):
        sc = scenes.box_room(width=4, height=4)
        sc['render_setting']['bvh_leaf_size'] = leaf
        small[leaf] = vb.Scene(host_ctx, sc).build_accel().info()['bvh_node_count']
    assert small['auto'] == small[3]
    for key, value in (('bvh_collapse', 'binned'), ('bvh_leaf_size', 4), ('bvh_leaf_size', 0),
                       ('bvh_leaf_size', 'large')):
        sc = scenes.box_room(width=4, height=4)
        sc['render_setting'][key] = value
        with pytest.raises(vb.UnsupportedError, match=key):
            vb.Scene(host_ctx, sc)


@pytest.mark.parametrize('kind, ok', [('linear', True), ('aces', True), ('reinhard', True), ('filmic', False)])
def test_tone_mapper_parse(vb, host_ctx, kind, ok):
    sc = scenes.box_room(width=4, height=4)
    sc['camera']['param']['radiance_collector']['param']['tone_mapper'] = {'type': kind}
    if ok:
        vb.Scene(host_ctx, sc)
    else:
        with pytest.raises(vb.UnsupportedError, match='tone mapper'):
            vb.Scene(host_ctx, sc)


def test_point_and_spot_light_records(vb, host_ctx):
    # PointLight / SpotLight (point.cpp:20-43, spot.cpp:19-70): appended after
    # the area light; spot angles clamped and turned into cosines; powers
    # 4 pi avg and 2 pi avg (1 - (2 angle + falloff) / 2), angles in radians.
    s = vb.Scene(host_ctx, scenes.point_light_room(8, 8, light_sampler='power'))
    L = s.export('lights', np.float32).reshape(-1, 28)
    U = L.view(np.uint32)
    assert L.shape[0] == 3 and list(U[:, 16]) == [0, 1, 2]
    np.testing.assert_allclose(L[1, 20:23], [-0.2, 0.9, 0.1])
    d = np.array([-0.3, -1.0, -0.4]) / np.linalg.norm([-0.3, -1.0, -0.4])
    np.testing.assert_allclose(L[2, 24:27], d, rtol=1e-6)
    a, f = math.radians(30.0), math.radians(12.0)
    np.testing.assert_allclose(L[2, 17:19], [math.cos(a), math.cos(a - f)], rtol=1e-6)
    y = lambda rgb: 0.212671 * rgb[0] + 0.715160 * rgb[1] + 0.072169 * rgb[2]
    np.testing.assert_allclose(L[1, 7], y(L[1, 12:15]) * 4 * math.pi, rtol=1e-5)
    np.testing.assert_allclose(L[2, 7], y(L[2, 12:15]) * 2 * math.pi * (1 - 0.5 * (2 * a + f)), rtol=1e-5)
    # The power sampler's pmf follows those powers.
    pmf = s.export('light_pmf', np.float32)
    np.testing.assert_allclose(pmf, L[:, 7] / L[:, 7].sum(), rtol=1e-5)


def test_rt_integrator_takes_delta_and_environment_lights(vb, host_ctx):
    # ReSTIR DI draws its candidates through the generic light sampler, so
    # point, spot and environment lights load with the rt integrator.
    sc = scenes.point_light_room(8, 8, dimension=3)
    sc['integrator'] = {'type': 'rt', 'param': {'max_depth': 4}}
    sc['light_sampler']['param']['lights'].append(scenes.large_scene()['light_sampler']['param']['lights'][0])
    sc['light_sampler']['param']['lights'][-1]['param']['color']['node']['param'].update(width=32, height=16)
    s = vb.Scene(host_ctx, sc)
    assert s.info()['light_count'] == 3  # the area light, the point and the spot
    # The light sampler draws over those and the sky.
    assert s.export('integrator', np.uint32)[9] == 4


def test_default_spectrum_is_srgb(vb, host_ctx):
    # SpectrumDesc::init defaults to "srgb" (node_desc.cpp:347-350): three RGB
    # channels, colours stored as RGB rather than sigmoid coefficients.
    sc = scenes.box_room(width=4, height=4)
    sc.pop('spectrum')
    s = vb.Scene(host_ctx, sc)
    assert s.info()['spectrum_dim'] == 3
    integ = s.export('integrator', np.uint32)
    assert integ[10] == 1
    mats = s.export('materials', np.float32).reshape(-1, 16)
    left = [m for m in sc['materials'] if m['name'] == 'LeftWall'][0]['param']['color']
    np.testing.assert_allclose(mats[3, 4:7], left, rtol=1e-6)
    hero = vb.Scene(host_ctx, scenes.box_room(width=4, height=4))
    assert hero.export('integrator', np.uint32)[10] == 0
    sc['spectrum'] = {'type': 'spectral_upsampling'}
    with pytest.raises(vb.UnsupportedError, match='spectrum'):
        vb.Scene(host_ctx, sc)


def test_sphere_matches_reference_tessellation(vb, host_ctx):
    # Sphere (sphere.cpp:17-87): 2 + (n - 1) * 2n vertices on the sphere,
    # 2n + (n - 2) * 4n + 2n triangles, every one facing outwards.
    n, R = 6, 0.25
    sc = scenes.box_room(width=4, height=4)
    sc['shapes'].append({'type': 'sphere', 'name': 'ball', 'param': {
        'radius': R, 'sub_div': n, 'material': 'TallBox',
        'transform': {'type': 'trs', 'param': {'t': [0.0, 0.3, 0.0]}}}})
    s = vb.Scene(host_ctx, sc)
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    nv, nt = 2 + (n - 1) * 2 * n, 2 * n + (n - 2) * 4 * n + 2 * n
    ball_p = pos[-nv:] - [0.0, 0.3, 0.0]
    np.testing.assert_allclose(np.linalg.norm(ball_p, axis=1), R, rtol=1e-5)
    tris = idx[-nt:] - (len(pos) - nv)
    assert tris.min() == 0 and tris.max() == nv - 1
    p = ball_p[tris]
    ng = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    assert np.all(np.einsum('ij,ij->i', ng, p.mean(1)) > 0)
    # The reference's first fan triangle and first band triangle.
    np.testing.assert_array_equal(tris[0], [0, 2, 1])
    np.testing.assert_array_equal(tris[2 * n], [1, 2, 1 + 2 * n])
