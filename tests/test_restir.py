"""Real-time ReSTIR integrator ("rt"): scene-schema parsing of its settings,
the per-frame parameter block, and host-side checks of the oracle's ReSTIR
restatement (motion vectors, reservoir invariants, determinism)."""
import math

import numpy as np
import pytest

import oracle
from vision_b200 import scenes

PARAM_U32 = dict(di_open=0, di_spatial=1, di_s_count=2, di_temporal=3, di_history=4, di_t_count=5, di_t_mis=6,
                 di_max_age=7, gi_open=16, gi_spatial=17, gi_s_count=18, gi_temporal=19, gi_history=20,
                 M_light=32, M_bsdf=33, max_recursion=34, pairwise=35, gi_max_depth=36, frame=37, width=38, height=39)
PARAM_F32 = dict(di_diff=8, di_s_dot=9, di_s_depth=10, di_s_radius=11, di_t_dot=12, di_t_depth=13, di_t_radius=14)


def _rt_scene(w=48, h=32, direct=None, indirect=None, max_depth=4, **kw):
    sc = scenes.box_room(w, h, dimension=3, **kw)
    sc['integrator'] = {'type': 'rt', 'param': {'max_depth': max_depth, 'min_depth': 5,
                                                 'direct': direct or {}, 'indirect': indirect or {}}}
    return sc


def _fields(p):
    u = p.view('<u4')
    f = p.view('<f4')
    out = {k: int(u[i]) for k, i in PARAM_U32.items()}
    out.update({k: float(f[i]) for k, i in PARAM_F32.items()})
    m = f[40:56].reshape(4, 4)   # w2c, column-major
    out['w2c'] = m.T.copy()
    out['view_pos'] = f[104:107].copy()
    out['prev_view_pos'] = f[107:110].copy()
    return out


def test_rt_defaults_follow_reference(vb, host_ctx):
    # SpatialResamplingParam / TemporalResamplingParam defaults (ReSTIR/common.h:19-67),
    # ReSTIRDI (direct.cpp:9-15), RealTimeIntegrator max_depth - 1 (rt.cpp:30).
    s = vb.Scene(host_ctx, _rt_scene(max_depth=16)).build_accel()
    p = _fields(s.restir_params(0))
    assert (p['M_light'], p['M_bsdf'], p['max_recursion'], p['pairwise']) == (10, 1, 5, 0)
    assert (p['di_spatial'], p['di_s_count'], p['di_temporal'], p['di_history'], p['di_t_count']) == (1, 1, 1, 5, 9)
    assert p['di_max_age'] == 30 and p['di_open'] == 1 and p['gi_open'] == 1
    assert p['gi_max_depth'] == 15
    np.testing.assert_allclose(p['di_s_dot'], math.cos(math.radians(35.0)), rtol=1e-6)
    np.testing.assert_allclose(p['di_t_dot'], math.cos(math.radians(35.0)), rtol=1e-6)
    np.testing.assert_allclose([p['di_diff'], p['di_s_depth'], p['di_s_radius'], p['di_t_depth'], p['di_t_radius']],
                               [0.3, 0.3, 30.0, 0.3, 8.0], rtol=1e-6)


def test_rt_settings_parse(vb, host_ctx):
    sc = _rt_scene(direct={'M_light': 32, 'M_bsdf': 2, 'pairwise': True, 'max_recursion': 6,
                           'spatial': {'theta': 5, 'radius': 20, 'sample_num': 5},
                           'temporal': {'history_limit': 20, 'theta': 2, 'N': 4}},
                   indirect={'open': False, 'spatial': {'open': False, 'sample_num': 7}})
    s = vb.Scene(host_ctx, sc).build_accel()
    p = _fields(s.restir_params(9))
    assert (p['M_light'], p['M_bsdf'], p['pairwise'], p['max_recursion']) == (32, 2, 1, 6)
    assert (p['di_s_count'], p['di_history'], p['di_t_count'], p['frame']) == (5, 20, 4, 9)
    np.testing.assert_allclose(p['di_s_dot'], math.cos(math.radians(5.0)), rtol=1e-6)
    np.testing.assert_allclose(p['di_t_dot'], math.cos(math.radians(2.0)), rtol=1e-6)
    # A closed spatial pass keeps sample_num = 1 (common.h:30).
    assert (p['gi_open'], p['gi_spatial'], p['gi_s_count']) == (0, 0, 1)


def test_rt_params_camera(vb, host_ctx):
    s = vb.Scene(host_ctx, _rt_scene()).build_accel()
    c2w = scenes.camera_c2w((0.1, 0.45, 1.7), (0.0, 0.5, 0.0))
    s.set_camera(c2w, 40.0)
    p = _fields(s.restir_params(0))
    np.testing.assert_allclose(p['w2c'], np.linalg.inv(c2w.astype(np.float64)), atol=2e-6)
    np.testing.assert_allclose(p['view_pos'], c2w[:3, 3], atol=1e-7)
    # No frame rendered yet: the previous camera is the current one.
    np.testing.assert_allclose(p['prev_view_pos'], c2w[:3, 3], atol=1e-7)
    assert (p['width'], p['height']) == (48, 32)


@pytest.mark.parametrize('change, needle', [
    (lambda sc: sc['spectrum']['param'].update(dimension=4), 'hero dimension'),
    (lambda sc: sc['integrator']['param']['direct'].update(spatial={'sample_num': 17}), 'sample_num'),
    (lambda sc: sc['integrator']['param'].update(max_depth=2), 'max_depth'),
])
def test_rt_rejects_unsupported(vb, host_ctx, change, needle):
    sc = _rt_scene()
    change(sc)
    with pytest.raises(vb.UnsupportedError, match=needle):
        vb.Scene(host_ctx, sc)


def test_restir_needs_device_and_rt(vb, host_ctx):
    s = vb.Scene(host_ctx, _rt_scene()).build_accel()
    with pytest.raises(vb.VisionError):
        s.restir_frame(0, 0)
    plain = vb.Scene(host_ctx, scenes.box_room(16, 16, dimension=3)).build_accel()
    with pytest.raises(vb.VisionError, match='rt'):
        plain.restir_params(0)


def _oracle_frames(vb, ctx, sc, cams, w, h, threads=4):
    s = vb.Scene(ctx, sc).build_accel()
    o = oracle.OracleScene(s)
    ort = oracle.OracleRestir(o, w, h)
    prev = None
    for f, c2w in enumerate(cams):
        s.set_camera(c2w, 40.0)
        p = s.restir_params(f)
        if prev is not None:
            # The library would take the previous frame's camera after a real
            # frame; a host-only context renders none, so patch it in here.
            pv = prev.view('<f4')
            pp = p.view('<f4')
            pp[56:72] = pv[40:56]            # prev_w2c <- w2c
            pp[72:104] = prev_cam.view('<f4')  # prev_cam
            pp[107:110] = pv[104:107]        # prev_view_pos
        prev_cam = s.export('camera').copy()
        ort.frame(s.export('camera'), p, 0, threads)
        prev = p
        yield s, ort, p


def test_oracle_static_camera_motion_is_zero(vb, host_ctx):
    sc = scenes.many_lights(40, 30, emitters=60, seed=2, M_light=4, max_depth=3)
    c2w = scenes.camera_c2w((0.0, 0.5, 1.85), (0.0, 0.5, 0.0))
    for s, ort, p in _oracle_frames(vb, host_ctx, sc, [c2w] * 3, 40, 30):
        pass
    mv = ort.buffer('motion', np.dtype(('<f4', 2)))
    surf = ort.buffer('surfaces', vb.RT_SURFACE_DTYPE)
    hit = surf['hit']['inst_id'] != 0xffffffff
    assert hit.mean() > 0.5
    assert np.abs(mv[hit]).max() < 1e-3
    r = ort.buffer('di_reservoirs', vb.DI_RESERVOIR_DTYPE)
    assert np.all(r['W'][hit] >= 0.0) and np.all(np.isfinite(r['W']))
    # Temporal history is capped at C <= history_limit * C_canonical (20), and
    # spatial reuse adds at most 5 neighbours of the same cap.
    assert r['C'].max() <= 21.0 * 6
    gi = ort.buffer('gi_reservoirs', vb.GI_RESERVOIR_DTYPE)
    assert np.all(np.isfinite(gi['W'][hit]))


def test_oracle_moving_camera_motion_vectors(vb, host_ctx):
    # FrameBuffer::compute_motion_vec: p_film minus the previous camera's
    # raster position of the surface point; checked against numpy projection.
    sc = scenes.many_lights(40, 30, emitters=30, seed=2, M_light=2, max_depth=3, gi=False)
    cams = scenes.camera_spline(2, seed=5)
    frames = list(_oracle_frames(vb, host_ctx, sc, cams, 40, 30))
    s, ort, p = frames[-1]
    mv = ort.buffer('motion', np.dtype(('<f4', 2)))
    surf = ort.buffer('surfaces', vb.RT_SURFACE_DTYPE)
    hit = (surf['hit']['inst_id'] != 0xffffffff) & (surf['is_replaced'] == 0)
    pos = surf['pos'][hit].astype(np.float64)
    prev_w2c = np.linalg.inv(cams[0].astype(np.float64))
    c = pos @ prev_w2c[:3, :3].T + prev_w2c[:3, 3]
    a, b = c[:, 0] / c[:, 2], c[:, 1] / c[:, 2]
    cam = s.export('camera').view('<f4')
    tan, lo_x, hi_y, span_x, span_y = cam[16:21]
    rx = (a / tan - lo_x) / span_x * 40
    ry = (hi_y - b / tan) / span_y * 30
    ys, xs = np.nonzero(hit)
    # p_film = pixel centre + box-filter jitter (|jitter| <= 0.5).
    film_x = rx + mv[hit][:, 0]
    film_y = ry + mv[hit][:, 1]
    assert np.all(np.abs(film_x - (xs + 0.5)) <= 0.5 + 1e-3)
    assert np.all(np.abs(film_y - (ys + 0.5)) <= 0.5 + 1e-3)
    assert np.abs(mv[hit]).max() > 0.05  # the camera did move


def test_oracle_restir_deterministic(vb, host_ctx):
    sc = scenes.many_lights(32, 24, emitters=40, seed=4, M_light=4, max_depth=3)
    cams = scenes.camera_spline(3, seed=1)
    a = [ort.buffer('film', np.dtype(('<f4', 4))).copy() for _, ort, _ in _oracle_frames(vb, host_ctx, sc, cams, 32, 24, 1)]
    b = [ort.buffer('film', np.dtype(('<f4', 4))).copy() for _, ort, _ in _oracle_frames(vb, host_ctx, sc, cams, 32, 24, 4)]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_oracle_restir_direct_light_is_unbiased_for_environment_and_delta_lights(vb, host_ctx):
    # ReSTIR DI draws light candidates through the generic light sampler: the
    # environment (map coordinates, solid-angle pdf), point and spot lights
    # (MIS weight 1 / M_light) beside area lights, and BSDF candidates that
    # escape to the environment.  With temporal and spatial reuse off, a frame
    # is an unbiased estimate of the direct light at the primary hit, so its
    # mean over frames must match the path tracer at max_depth 1 with light
    # sampling only (mis_mode 1), up to noise (a z-test on the image mean).
    import copy
    w, h, frames = 48, 32, 200
    sc = scenes.many_lights(w, h, emitters=20, seed=5, M_light=4, max_depth=4, gi=False)
    sc['shapes'] = [x for x in sc['shapes'] if x['name'] != 'back']
    sc['light_sampler']['param']['lights'] = [{'type': 'spherical', 'param': {
        'color': {'channels': 'xyz', 'node': {'type': 'sky', 'param': {
            'width': 64, 'height': 32, 'sun_elevation': 20.0, 'sun_azimuth': 180.0, 'sun_radius': 8.0,
            'sun_peak': 40.0}}}, 'scale': 1.0}}] + scenes.point_light_room()['light_sampler']['param']['lights']
    d = sc['integrator']['param']['direct']
    d['spatial'] = {'open': False}
    d['temporal'] = {'open': False}
    s = vb.Scene(host_ctx, sc).build_accel()
    ort = oracle.OracleRestir(oracle.OracleScene(s), w, h)
    cam = s.export('camera').copy()
    means, acc, picked = [], 0.0, set()
    for f in range(frames):
        ort.frame(cam, s.restir_params(f), 0, 4)
        x = ort.buffer('di_radiance', np.dtype(('<f4', 4)))[..., :3]
        means.append(x.mean())
        picked |= set(np.unique(ort.buffer('di_reservoirs', vb.DI_RESERVOIR_DTYPE)['light_index']).tolist())
    n_lights = s.export('integrator', np.uint32)[9]
    # Reservoirs chose the sky (the last light), the point and the spot light.
    assert {n_lights - 1, n_lights - 2, n_lights - 3} <= picked
    pt = copy.deepcopy(sc)
    pt['integrator'] = {'type': 'pt', 'param': {'max_depth': 1, 'min_depth': 5, 'rr_threshold': 1.0, 'mis_mode': 1}}
    ref = oracle.OracleScene(vb.Scene(host_ctx, pt).build_accel()).render(0, 1024, threads=4)[..., :3].mean()
    rt, se = np.mean(means), np.std(means) / np.sqrt(frames)
    assert abs(rt - ref) <= 4.0 * se + 0.003 * ref, (rt, ref, se)
