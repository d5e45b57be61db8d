"""Parity on the configurations the benchmark times.

The bench renders with the PCG sampler, on the full 2,327,680-triangle large
scene at 1024 x 1024 and runs ReSTIR at 1920 x 1080 with 10,000 emitters, 32
light candidates and a 30-pixel spatial radius.  These tests check the CUDA
path against the oracle on exactly those inputs: the device sampler streams
bit for bit, closest hits on the benchmarked BVH bit for bit, matched-seed
images of the box room and of windows of the large scene (per-pixel z-test
from FP64 sums and sums of squares on both sides), and ReSTIR frames at the
benchmark's parameters."""
import numpy as np
import pytest

import oracle
from helpers import mean_z, path_sums, pixel_z, seeded_rays
from vision_b200 import scenes

pytestmark = pytest.mark.gpu


def _pcg32_floats(initstate, initseq, n):
    # PCG32 (O'Neill 2014) pcg32_srandom_r / pcg32_random_r, written out in
    # Python integers; the sampler's float is the top 24 output bits / 2^24.
    mult, mask = 6364136223846793005, (1 << 64) - 1
    inc = ((initseq << 1) | 1) & mask
    state = ((inc + initstate) * mult + inc) & mask
    out = []
    for _ in range(n):
        xs = (((state >> 18) ^ state) >> 27) & 0xffffffff
        rot = state >> 59
        r = ((xs >> rot) | (xs << ((-rot) & 31))) & 0xffffffff
        state = (state * mult + inc) & mask
        out.append((r >> 8) / 16777216.0)
    return np.array(out, np.float32)


@pytest.mark.parametrize('kind, seed', [(0, 0), (1, 0), (1, 1), (1, 7)])
def test_device_sampler_streams_bit_exact(vb, gpu_ctx, kind, seed):
    rng = np.random.default_rng(100 + kind * 10 + seed)
    keys = rng.integers(0, 1 << 32, size=(2048, 4), dtype=np.uint64).astype(np.uint32)
    keys[:, 0] %= 1024
    keys[:, 1] %= 1024
    # Stream starts the renderer uses: the wavelength stream (dim 0xffffffff)
    # and the main stream (dim 0) of the first and last pixels and frames.
    fixed = np.array([[0, 0, 0, 0], [0, 0, 0, 0xffffffff], [1023, 1023, 63, 0], [1023, 1023, 63, 0xffffffff],
                      [255, 0, 15, 0], [0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff]], np.uint32)
    keys = np.concatenate([fixed, keys])
    draws = 96
    got = vb.sampler_stream(gpu_ctx, keys, draws, kind=kind, seed=seed)
    for i, (px, py, sample, dim) in enumerate(keys):
        want = oracle.sampler_stream(int(px), int(py), int(sample), int(dim), draws, kind=kind, seed=seed)
        assert np.array_equal(got[i].view(np.uint32), want.view(np.uint32)), (i, keys[i])
    if kind == 1:
        for i in range(len(fixed)):
            px, py, sample, dim = (int(x) for x in keys[i])
            init = oracle.tea(oracle.tea(px, py), oracle.tea(sample, dim))
            assert np.array_equal(got[i], _pcg32_floats(init, seed, draws))
        # Draws cover [0, 1) (a truncated state would confine them).
        assert got.min() < 1e-3 and got.max() > 0.999 and abs(got.mean() - 0.5) < 0.01


def test_matched_seed_parity_pcg_box_room(vb, gpu_ctx):
    # The box-room benchmark configuration (PCG sampler, 4 hero wavelengths,
    # depth 8) at 64 x 64, 16 spp.
    sc = scenes.box_room(width=64, height=64, sampler='pcg')
    s = vb.Scene(gpu_ctx, sc).build_accel()
    o = oracle.OracleScene(s)
    s.render(0, 16, fp64=True)
    g = s.film()
    gs, gq = s.film(vb.FILM_SUM64), s.film(vb.FILM_SUMSQ64)
    pix = np.arange(64 * 64, dtype=np.uint32)
    cs, cq = path_sums(o.paths(pix, 0, 16))
    cs, cq = cs.reshape(64, 64, 3), cq.reshape(64, 64, 3)
    c = cs / 16.0
    assert np.all(np.isfinite(g))
    close = (np.abs(g[..., :3] - c) <= 1e-3 * (1.0 + np.abs(c))).all(-1)
    # Measured bar: per-pixel agreement as for the TEA/LCG box room.
    assert close.mean() >= 0.97, close.mean()
    z = pixel_z(gs[..., :3], gq[..., :3], 16, cs, cq, 16)
    assert (np.abs(z) > 4.0).mean() <= 0.002, np.sort(np.abs(z).ravel())[-10:]
    assert abs(g[..., :3].mean() - c.mean()) < 2e-3 * c.mean()


@pytest.mark.parametrize('sampler', ['independent', 'pcg'])
def test_independent_seeds_per_pixel_z_test(vb, gpu_ctx, sampler):
    # Frames 0..63 on the GPU against frames 64..127 on the oracle:
    # independent samples of one estimator.  The per-pixel z statistic from
    # each side's own sums and sums of squares is then close to N(0, 1).
    s = vb.Scene(gpu_ctx, scenes.box_room(width=32, height=32, sampler=sampler)).build_accel()
    o = oracle.OracleScene(s)
    s.render(0, 64, fp64=True)
    gs, gq = s.film(vb.FILM_SUM64)[..., :3], s.film(vb.FILM_SUMSQ64)[..., :3]
    np.testing.assert_array_equal(s.film(vb.FILM_SUM64)[..., 3], 64.0)
    cs, cq = path_sums(o.paths(np.arange(32 * 32, dtype=np.uint32), 64, 64))
    z = pixel_z(gs, gq, 64, cs.reshape(32, 32, 3), cq.reshape(32, 32, 3), 64)
    assert np.all(np.isfinite(z))
    assert abs(z.mean()) < 0.1, z.mean()
    assert 0.7 < z.std() < 1.3, z.std()
    assert (np.abs(z) > 4.0).mean() < 0.005


_LARGE = {}


def _large_scene(vb, ctx):
    # The benchmarked scene, built once per session (2.3 M triangles).
    if 'scene' not in _LARGE:
        s = vb.Scene(ctx, scenes.large_scene()).build_accel()
        _LARGE['scene'] = s
        _LARGE['oracle'] = oracle.OracleScene(s)
    return _LARGE['scene'], _LARGE['oracle']


def test_full_large_scene_closest_hit_bit_exact(vb, gpu_ctx):
    s, o = _large_scene(vb, gpu_ctx)
    info = s.info()
    assert info['prim_count'] == 2327680
    pos = s.export('pos', np.float32).reshape(-1, 3)
    idx = s.export('idx', np.uint32).reshape(-1, 3)
    rng = np.random.default_rng(33)
    # Edge midpoints and vertices of a random subset of triangles, half of
    # them on the sphere, provoke ties between neighbouring triangles.
    sphere = np.where(s.export('prim_inst', np.uint32) == 0)[0]
    pick = np.concatenate([rng.choice(sphere, 20000, replace=False), rng.choice(len(idx), 20000, replace=False)])
    from helpers import edge_targets
    tg = edge_targets(pos, idx[pick])
    n = 1 << 20
    rays = np.concatenate([
        seeded_rays(n // 2, [-1.6, 0.05, -1.6], [1.6, 2.6, 1.6], seed=41, targets=tg),
        seeded_rays(n // 4, [-20.0, 0.05, -20.0], [20.0, 4.0, 20.0], seed=42, targets=tg),
        _camera_rays(s, n // 4, seed=43)])
    h_gpu, t_gpu = s.trace_closest(rays)
    h_cpu, t_cpu = o.trace_closest(rays)
    hit = h_cpu[:, 0] != 0xffffffff
    assert 0.3 < hit.mean() < 0.95, hit.mean()
    assert np.array_equal(h_gpu, h_cpu)
    assert np.array_equal(t_gpu.view(np.uint32), t_cpu.view(np.uint32))
    occ_gpu = s.trace_any(rays[:n // 4])
    occ_cpu = o.trace_any(rays[:n // 4])
    assert np.array_equal(occ_gpu, occ_cpu)


def _camera_rays(s, n, seed):
    # Rays from the benchmark camera's position (0, 2.2, 5) towards random
    # points around the sphere and the ground in front of it.
    rng = np.random.default_rng(seed)
    eye = np.array([0.0, 2.2, 5.0], np.float32)
    tgt = np.array([-3.0, -0.2, -3.0]) + np.array([6.0, 2.4, 6.0]) * rng.random((n, 3))
    d = (tgt - eye).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = eye
    rays[:, 4:7] = d
    rays[:, 7] = 3.0e38
    return rays


@pytest.mark.parametrize('window', [(464, 400), (200, 640)])
def test_large_scene_window_parity(vb, gpu_ctx, window):
    # A 96 x 96 window of the benchmark's 1024 x 1024 image at 16 spp, matched
    # seeds (PCG, full depth 16): (464, 400) sits on the displaced sphere and
    # its reflections, (200, 640) on the ground tiles and the horizon.
    s, o = _large_scene(vb, gpu_ctx)
    s.render(0, 16, fp64=True)
    x0, y0 = window
    k = 96
    gs = s.film(vb.FILM_SUM64)[y0:y0 + k, x0:x0 + k, :3]
    gq = s.film(vb.FILM_SUMSQ64)[y0:y0 + k, x0:x0 + k, :3]
    yy, xx = np.mgrid[y0:y0 + k, x0:x0 + k]
    pix = (yy * 1024 + xx).astype(np.uint32).ravel()
    cs, cq = path_sums(o.paths(pix, 0, 16))
    cs, cq = cs.reshape(k, k, 3), cq.reshape(k, k, 3)
    g, c = gs / 16.0, cs / 16.0
    assert np.all(np.isfinite(g)) and c.mean() > 0
    close = (np.abs(g - c) <= 2e-3 * (1.0 + np.abs(c))).all(-1)
    assert close.mean() >= 0.85, close.mean()
    z = pixel_z(gs, gq, 16, cs, cq, 16)
    assert (np.abs(z) > 4.0).mean() <= 0.005, np.sort(np.abs(z).ravel())[-10:]
    # The window means: a handful of paths that reach the sun (peak 5e4)
    # dominate them, so the bar is on their difference in standard errors.
    assert abs(mean_z(gs, gq, 16, cs, cq, 16)) < 4.0, (g.mean(), c.mean())


def test_restir_at_benchmark_parameters(vb, gpu_ctx):
    # The many-light benchmark frame: 1920 x 1080, 10,000 blackbody emitters,
    # power light sampler, 32 light candidates, temporal cap 20, 5 spatial
    # neighbours within 30 px, PCG sampler; three frames of its camera spline.
    w, h = 1920, 1080
    sc = scenes.many_lights(w, h)
    s = vb.Scene(gpu_ctx, sc).build_accel()
    o = oracle.OracleScene(s)
    ort = oracle.OracleRestir(o, w, h)
    F4 = np.dtype(('<f4', 4))
    for f, c2w in enumerate(scenes.camera_spline(64, seed=3)[:3]):
        s.set_camera(c2w, 40.0)
        params = s.restir_params(f)
        cam = s.export('camera').copy()
        # A new camera restarts the film: each frame is film sample 0.
        s.restir_frame(f, 0)
        ort.frame(cam, params, 0)
        gs, cs = s.restir_buffer('surfaces'), ort.buffer('surfaces', vb.RT_SURFACE_DTYPE)
        hit_eq = (gs['hit']['prim_id'] == cs['hit']['prim_id'])
        assert hit_eq.mean() >= 0.999, (f, hit_eq.mean())
        hit = cs['hit']['inst_id'] != 0xffffffff
        gd, cd = s.restir_buffer('di_radiance')[..., :3], ort.buffer('di_radiance', F4)[..., :3]
        gg, cg = s.restir_buffer('gi_radiance')[..., :3], ort.buffer('gi_radiance', F4)[..., :3]
        assert np.all(np.isfinite(gd)) and np.all(np.isfinite(gg))
        tol = lambda a, b: np.abs(a - b) <= 1e-4 + 2e-3 * np.abs(b)
        di_ok, gi_ok = tol(gd, cd).all(-1).mean(), tol(gg, cg).all(-1).mean()
        assert di_ok >= 0.99, (f, di_ok)
        assert gi_ok >= 0.98, (f, gi_ok)
        assert abs(gd.mean() - cd.mean()) <= 0.005 * cd.mean(), (f, gd.mean(), cd.mean())
        assert abs(gg.mean() - cg.mean()) <= 0.01 * cg.mean(), (f, gg.mean(), cg.mean())
        gr = s.restir_buffer('di_reservoirs')
        cr = ort.buffer('di_reservoirs', vb.DI_RESERVOIR_DTYPE)
        assert (gr['light_index'] == cr['light_index'])[hit].mean() >= 0.99
        gf, cf = s.film()[..., :3], ort.buffer('film', F4)[..., :3]
        assert tol(gf, cf).all(-1).mean() >= 0.98, f


@pytest.mark.parametrize('case', ['box_room', 'material_room', 'large_scene_small'])
def test_parity_against_the_oracles_own_scene(vb, gpu_ctx, case):
    # The oracle here builds the scene from the document itself
    # (oracle/scene.py), so nothing of the library's scene layer is shared
    # with the checker: matched seeds, per-pixel z-test and the image means.
    if case == 'box_room':
        sc = scenes.box_room(width=48, height=48, sampler='pcg')
    elif case == 'material_room':
        sc = scenes.material_room(48, 48, sampler='pcg')
    else:
        sc = scenes.large_scene(width=48, height=48, subdivisions=4, grid=60, tiles=4, sky_width=256,
                                sky_height=128)
    s = vb.Scene(gpu_ctx, sc).build_accel()
    o = oracle.OracleScene.from_json(sc)
    n = 32
    s.render(0, n, fp64=True)
    gs, gq = s.film(vb.FILM_SUM64)[..., :3], s.film(vb.FILM_SUMSQ64)[..., :3]
    cs, cq = path_sums(o.paths(np.arange(48 * 48, dtype=np.uint32), 0, n))
    cs, cq = cs.reshape(48, 48, 3), cq.reshape(48, 48, 3)
    z = pixel_z(gs, gq, n, cs, cq, n)
    assert (np.abs(z) > 4.0).mean() <= 0.005, np.sort(np.abs(z).ravel())[-10:]
    assert abs(mean_z(gs, gq, n, cs, cq, n)) < 4.0
    close = (np.abs(gs - cs) / n <= 2e-3 * (1.0 + np.abs(cs) / n)).all(-1).mean()
    assert close >= {'box_room': 0.97, 'material_room': 0.85, 'large_scene_small': 0.80}[case], close
