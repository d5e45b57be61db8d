"""SVGF denoiser of the real-time frame: the oracle's restatement of the
reference's passes (src/render_core/denoisers/SVGF/) on the host, and the
settings block the library reads from the integrator's "denoiser" node."""
import numpy as np
import pytest

import oracle
from vision_b200 import scenes


def _scene(w=40, h=30, emitters=40):
    sc = scenes.many_lights(w, h, emitters=emitters, seed=3, M_light=4, max_depth=4)
    sc['integrator']['param']['denoiser'] = {'type': 'svgf', 'param': {'N': 3}}
    return sc


def test_denoiser_settings(vb, host_ctx):
    s = vb.Scene(host_ctx, _scene())
    p = s.denoiser_params()
    # The reference's defaults (svgf.h:41-51).
    assert (p['N'], p['history_limit'], p['moments_radius'], p['reproject'], p['filter_moments']) == (3, 32, 3, 1, 1)
    np.testing.assert_allclose([p['alpha'], p['moments_alpha'], p['sigma_rt'], p['sigma_normal']],
                               [0.05, 0.2, 10.0, 30.0])
    sc = _scene()
    sc['integrator']['param']['denoiser']['param'].update(N=5, alpha=0.1, sigma_rt=4.0, moments_filter_radius=2)
    p = vb.Scene(host_ctx, sc).denoiser_params()
    assert (p['N'], p['moments_radius']) == (5, 2)
    np.testing.assert_allclose([p['alpha'], p['sigma_rt']], [0.1, 4.0])
    sc['integrator']['param']['denoiser'] = {'type': 'oidn', 'param': {}}
    with pytest.raises(vb.UnsupportedError, match='denoiser'):
        vb.Scene(host_ctx, sc)


def _frames(vb, ctx, sc, cams, radiance_fn):
    s = vb.Scene(ctx, sc).build_accel()
    i = s.info()
    ort = oracle.OracleRestir(oracle.OracleScene(s), i['width'], i['height'])
    sp = s.denoiser_params()
    prev = None
    for f, c2w in enumerate(cams):
        s.set_camera(c2w, 40.0)
        p = s.restir_params(f)
        if prev is not None:
            # A host-only context renders no frame, so the previous camera is
            # patched in as the library would keep it.
            pv, pp = prev[0].view('<f4'), p.view('<f4')
            pp[56:72] = pv[40:56]
            pp[72:104] = prev[1].view('<f4')
            pp[107:110] = pv[104:107]
        cam = s.export('camera').copy()
        ort.svgf(cam, p, sp, radiance_fn(ort, f, cam, p, sp))
        prev = (p, cam)
        yield f, ort


def test_oracle_svgf_keeps_a_constant_illumination(vb, host_ctx):
    # Radiance = albedo * 0.5 + emission demodulates to 0.5 everywhere; every
    # pass is a normalised weighted mean, so the output is the input.  The
    # room has no emitting surfaces (a point light instead: an emitter's zero
    # albedo would demodulate to 0 and pull its neighbours down) and uses RGB
    # transport (three hero wavelengths can give an albedo channel below
    # zero, which demodulation clamps).
    sc = _scene(48, 36, emitters=0)
    sc.pop('spectrum')
    sc['shapes'] = [x for x in sc['shapes'] if x['name'] != 'light']
    sc['light_sampler']['param']['lights'] = scenes.point_light_room()['light_sampler']['param']['lights'][:1]
    # The camera inside the room: every ray hits a wall.  (A miss keeps depth
    # -1 and a zero normal, which the reference's reprojection test accepts
    # beside a silhouette, so background pixels would feed in.)
    cams = [scenes.camera_c2w((0.0, 0.5, 0.45), (0.0, 0.45, -0.5))] * 3
    state = {}

    def radiance(ort, f, cam, p, sp):
        # This frame's albedo and emission, from a second oracle that runs the
        # same frame first (same camera, frame index and sampler streams).
        if 'probe' not in state:
            state['probe'] = oracle.OracleRestir(ort.oscene, ort.width, ort.height)
        probe = state['probe']
        probe.svgf(cam, p, sp, np.zeros((ort.height, ort.width, 4), np.float32))
        a = probe.buffer('svgf_albedo', np.dtype(('<f4', 4)))
        e = probe.buffer('svgf_emission', np.dtype(('<f4', 4)))
        rad = a * 0.5 + e
        rad[..., 3] = 1.0
        state['rad'] = rad
        return rad

    for f, ort in _frames(vb, host_ctx, sc, cams, radiance):
        out = ort.buffer('denoised', np.dtype(('<f4', 4)))[..., :3]
        geom = ort.buffer('gbuffer', vb.SVGF_GEOM_DTYPE)
        albedo = ort.buffer('svgf_albedo', np.dtype(('<f4', 4)))[..., :3]
        hit = geom['linear_depth'] >= 0
        assert hit.all() and albedo.min() >= 0.001
        np.testing.assert_allclose(out[hit], state['rad'][..., :3][hit], rtol=2e-5, atol=1e-6)
        hist = ort.buffer('svgf_history', np.dtype('<f4'))
        # Static camera: every surface pixel reprojects onto itself.
        assert (hist[hit] == f + 1).mean() > 0.99, (f, np.unique(hist[hit]))
        motion = ort.buffer('svgf_motion', np.dtype(('<f4', 2)))
        assert np.abs(motion[hit]).max() < 1e-3


def test_oracle_svgf_reduces_noise(vb, host_ctx):
    # Noisy frames of the real-time oracle with reuse off (independent
    # frames; ReSTIR's own reuse already smooths its frames), static camera:
    # after 24 frames the denoised frame is far closer to the 128-frame mean
    # than a raw frame is.  RGB transport: demodulation divides by the
    # albedo, and three hero wavelengths' RGB albedo is noisy itself.
    from scipy.ndimage import maximum_filter
    w, h = 32, 24
    sc = _scene(w, h)
    sc.pop('spectrum')
    for stage in ('direct', 'indirect'):
        sc['integrator']['param'][stage].update(spatial={'open': False}, temporal={'open': False})
    s = vb.Scene(host_ctx, sc).build_accel()
    rt = oracle.OracleRestir(oracle.OracleScene(s), w, h)
    c2w = scenes.camera_c2w((0.0, 0.5, 1.85), (0.0, 0.5, 0.0))
    s.set_camera(c2w, 40.0)
    frames = []
    for f in range(128):
        rt.frame(s.export('camera'), s.restir_params(f), 0, 8)
        frames.append(rt.buffer('film', np.dtype(('<f4', 4))).copy())
    ref = np.mean(frames, axis=0)[..., :3]

    def radiance(ort, f, cam, p, sp):
        return frames[f]

    # SVGF frame f denoises the real-time frame f (same camera jitter).  The
    # error is measured away from pixels where a camera ray met an emitter:
    # their jittered emission is added back unfiltered.
    emitted = np.zeros((h, w), bool)
    for f, ort in _frames(vb, host_ctx, sc, [c2w] * 24, radiance):
        emitted |= ort.buffer('svgf_emission', np.dtype(('<f4', 4)))[..., :3].max(-1) > 0
    clean = ~maximum_filter(emitted, size=3) & (ort.buffer('gbuffer', vb.SVGF_GEOM_DTYPE)['linear_depth'] >= 0)
    assert clean.mean() > 0.4
    den = ort.buffer('denoised', np.dtype(('<f4', 4)))[..., :3]
    err_raw = np.mean((frames[23][..., :3] - ref)[clean] ** 2)
    err_den = np.mean((den - ref)[clean] ** 2)
    # Measured: 0.108 raw against 0.0058 denoised.
    assert err_den < 0.15 * err_raw, (err_den, err_raw)
