"""SVGF denoiser on the GPU against the oracle's restatement along a moving
camera: both sides denoise the GPU's own film, so the G-buffer (normals,
depth, gradients, each material's albedo, emission, motion), the history
lengths and the denoised frame are compared pass for pass.  FP32 rounding of
exp / pow and of the interpolated normals can flip a rare reprojection
decision, so the bars are per-pixel agreement fractions."""
import numpy as np
import pytest

import oracle
from vision_b200 import scenes

pytestmark = pytest.mark.gpu

F4 = np.dtype(('<f4', 4))


def _close(a, b, rtol, atol):
    return np.abs(a - b) <= atol + rtol * np.abs(b)


def _materials(sc):
    # One surface of each material family, so the albedo of every lobe set
    # (MaterialEvaluator::albedo) is exercised.
    m = {x['name']: x for x in sc['materials']}
    m['TallBox'].update({'type': 'metal', 'param': {'material_name': 'Au', 'roughness': 0.3}})
    m['ShortBox'].update({'type': 'plastic', 'param': {'color': [0.1, 0.2, 0.7], 'roughness': 0.3}})
    m['Floor'].update({'type': 'principled_bsdf', 'param': {
        'color': [0.6, 0.5, 0.4], 'metallic': 0.3, 'roughness': 0.4, 'sheen_weight': 0.5, 'coat_weight': 0.4,
        'coat_roughness': 0.2}})
    m['BackWall'].update({'type': 'substrate', 'param': {'color': [0.5, 0.6, 0.4], 'roughness': 0.3}})
    m['LeftWall'].update({'type': 'mirror', 'param': {'color': [0.9, 0.8, 0.7], 'roughness': 0.3}})
    m['RightWall'].update({'type': 'glass', 'param': {'color': [1.0, 1.0, 1.0], 'roughness': 0.3, 'ior': 1.5}})


@pytest.mark.parametrize('spectrum', ['hero', 'srgb'])
def test_svgf_matches_oracle(vb, gpu_ctx, spectrum):
    w, h = 96, 64
    sc = scenes.many_lights(w, h, emitters=200, seed=5, M_light=8, spatial_radius=12.0, max_depth=4)
    sc['integrator']['param']['denoiser'] = {'type': 'svgf', 'param': {'N': 3}}
    _materials(sc)
    if spectrum == 'srgb':
        sc.pop('spectrum')
    s = vb.Scene(gpu_ctx, sc).build_accel()
    s.denoiser_enable(True)
    ort = oracle.OracleRestir(oracle.OracleScene(s), w, h)
    sp = s.denoiser_params()
    for f, c2w in enumerate(scenes.camera_spline(6, seed=3)):
        s.set_camera(c2w, 40.0)
        params = s.restir_params(f)
        cam = s.export('camera').copy()
        s.restir_frame(f, 0)
        ort.svgf(cam, params, sp, s.film())
        gg, cg = s.restir_buffer('gbuffer'), ort.buffer('gbuffer', vb.SVGF_GEOM_DTYPE)
        hit = cg['linear_depth'] >= 0
        assert hit.mean() > 0.5
        assert ((gg['linear_depth'] >= 0) == hit).mean() >= 0.999
        assert _close(gg['normal'], cg['normal'], 1e-4, 1e-5).all(-1)[hit].mean() >= 0.999
        assert _close(gg['linear_depth'], cg['linear_depth'], 1e-5, 1e-6)[hit].mean() >= 0.999
        assert _close(gg['fwidth'], cg['fwidth'], 1e-3, 1e-4)[hit].mean() >= 0.99
        assert _close(gg['depth_gradient'], cg['depth_gradient'], 1e-3, 1e-5)[hit].mean() >= 0.99
        assert np.array_equal(gg['p_film'], cg['p_film'])
        ga, ca = s.restir_buffer('svgf_albedo')[..., :3], ort.buffer('svgf_albedo', F4)[..., :3]
        assert _close(ga, ca, 1e-4, 1e-5).all(-1)[hit].mean() >= 0.995, f
        assert (ca[hit].max(-1) > 0).mean() > 0.3
        ge, ce = s.restir_buffer('svgf_emission')[..., :3], ort.buffer('svgf_emission', F4)[..., :3]
        assert _close(ge, ce, 1e-4, 1e-5).all(-1).mean() >= 0.999
        gm, cm = s.restir_buffer('svgf_motion'), ort.buffer('svgf_motion', np.dtype(('<f4', 2)))
        assert _close(gm, cm, 1e-3, 1e-3).all(-1).mean() >= 0.995
        gh, ch = s.restir_buffer('svgf_history'), ort.buffer('svgf_history', np.dtype('<f4'))
        assert (gh == ch).mean() >= 0.995, f
        if f > 0:
            assert (ch[hit] > 1).mean() > 0.5  # the moving camera still reprojects most pixels
        gd, cd = s.restir_buffer('denoised')[..., :3], ort.buffer('denoised', F4)[..., :3]
        assert np.all(np.isfinite(gd))
        ok = _close(gd, cd, 2e-3, 1e-4).all(-1).mean()
        # The bar leaves room for a rare flipped reprojection decision and its
        # filtered neighbourhood.
        assert ok >= 0.98, (f, ok)


def test_svgf_leaves_the_frame_alone(vb, gpu_ctx):
    # The denoiser reads the frame's film and writes its own output: the
    # ReSTIR frame and its film are the same with it on and off.
    w, h = 48, 32
    sc = scenes.many_lights(w, h, emitters=50, seed=2, M_light=4, max_depth=4)
    films = []
    for on in (False, True):
        s = vb.Scene(gpu_ctx, sc).build_accel()
        s.denoiser_enable(on)
        for f, c2w in enumerate(scenes.camera_spline(3, seed=1)):
            s.set_camera(c2w, 40.0)
            s.restir_frame(f, 0)
        films.append(s.film())
        if not on:
            with pytest.raises(vb.VisionError):
                s.restir_buffer('denoised')
    assert np.array_equal(films[0], films[1])
    den = s.restir_buffer('denoised')
    assert np.all(np.isfinite(den)) and den[..., 3].min() == 1.0
