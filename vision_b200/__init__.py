"""vision_b200 — B200-native spectral path-tracing hot path of FaithZL/Vision.

Python mirror of the reference's render entry (the SDK's VisionRenderer,
src/sdk/vision.h:66-99, and the fixed pipeline's prepare -> compile -> render
loop, src/pipelines/fixed/pipeline.cpp:9-44) over the C ABI of
libvision_b200.so (include/vision_b200.h).  There is no CPU fallback: if the
shared library is missing the import fails.
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# VISION_B200_LIB may name another build of the same library (for example one
# compiled with different floating-point contraction flags).
LIB_PATH = os.environ.get('VISION_B200_LIB') or os.path.join(HERE, 'libvision_b200.so')
TABLE_CACHE = os.path.join(HERE, 'data', 'srgb2spec_64.bin')

VS_OK = 0
VS_E_INVALID = 1
VS_E_UNSUPPORTED = 2
VS_E_PARSE = 3
VS_E_CUDA = 4
VS_E_STATE = 5
VS_E_NO_DEVICE = 6
VS_E_RANGE = 7

FILM_FP32 = 0
FILM_FP64 = 1
FILM_LINEAR = 0
FILM_EXPOSED = 1
FILM_SUM64 = 2
FILM_DISPLAY = 3
FILM_HDR = 4
FILM_RGBA8 = 5
FILM_SUMSQ64 = 6

EXPORT = dict(mesh_pos=27, mesh_idx=28, meshes=29, inst_mesh=30, inst_w2o=31,
              pos=0, nrm=1, uv=2, idx=3, prim_inst=4, instances=5, materials=6, lights=7, prim_alias=8,
              prim_pmf=9, light_alias=10, light_pmf=11, camera=12, integrator=13, spd=14, material_rgb=15,
              light_rgb=16, bvh_nodes=17, bvh_tris=18, luts=19, env=20, env_tex=21,
              env_marginal=22, env_marginal_func=23, env_cond=24, env_cond_func=25, rgb2spec=26,
              tex_texels=32, textures=33)


class VisionError(RuntimeError):
    def __init__(self, code, message):
        super().__init__('%s (status %d)' % (message, code))
        self.code = code


class UnsupportedError(VisionError):
    pass


class HitStruct(ctypes.Structure):
    _fields_ = [('inst_id', ctypes.c_uint32), ('prim_id', ctypes.c_uint32), ('u', ctypes.c_float), ('v', ctypes.c_float)]


class SceneInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        'vertex_count', 'prim_count', 'instance_count', 'material_count', 'light_count', 'prim_alias_count',
        'spd_floats', 'bvh_node_count', 'bvh_depth', 'width', 'height', 'spectrum_dim', 'max_depth', 'accel_built',
        'two_level', 'mesh_count')]


class JobDesc(ctypes.Structure):
    _fields_ = [('scene', ctypes.c_uint32), ('width', ctypes.c_uint32), ('height', ctypes.c_uint32),
                ('spp', ctypes.c_uint32), ('frame_begin', ctypes.c_uint32), ('fov_y_deg', ctypes.c_float),
                ('use_c2w', ctypes.c_int), ('c2w', ctypes.c_float * 16)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ('submitted', 'completed', 'batches', 'graph_launches',
                                               'kernel_launches')] + \
               [(n, ctypes.c_double) for n in ('paths', 'wall_s', 'gpu_busy_s', 'p50_ms', 'p95_ms', 'p99_ms',
                                               'mean_ms', 'max_ms')] + \
               [('peak_bytes', ctypes.c_uint64), ('peak_jobs', ctypes.c_uint32),
                ('resident_bytes', ctypes.c_uint64), ('scratch_bytes', ctypes.c_uint64)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError('libvision_b200.so not built: run `python vision_b200/build.py` (%s missing)' % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    U32 = ctypes.c_uint32
    sig = {
        'vs_version': ([], ctypes.c_int),
        'vs_context_create': ([ctypes.c_int, ctypes.POINTER(P)], ctypes.c_int),
        'vs_context_destroy': ([P], None),
        'vs_last_error': ([P], ctypes.c_char_p),
        'vs_scene_load_json': ([P, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_char_p,
                                ctypes.POINTER(P)], ctypes.c_int),
        'vs_scene_destroy': ([P], None),
        'vs_scene_build_accel': ([P], ctypes.c_int),
        'vs_set_resolution': ([P, U32, U32], ctypes.c_int),
        'vs_scene_add_instance': ([P, P, U32, P, U32, P, ctypes.c_char_p, ctypes.POINTER(U32)], ctypes.c_int),
        'vs_scene_clear_geometries': ([P], ctypes.c_int),
        'vs_scene_invalidate': ([P], ctypes.c_int),
        'vs_camera_set': ([P, P, ctypes.c_float], ctypes.c_int),
        'vs_scene_info_get': ([P, ctypes.POINTER(SceneInfo)], ctypes.c_int),
        'vs_scene_export_size': ([P, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
        'vs_scene_export': ([P, ctypes.c_int, P, ctypes.c_size_t], ctypes.c_int),
        'vs_render': ([P, U32, U32, ctypes.c_int, P], ctypes.c_int),
        'vs_synchronize': ([P], ctypes.c_int),
        'vs_film_download': ([P, P, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
        'vs_trace_closest_device': ([P, P, U32, P, P, P], ctypes.c_int),
        'vs_trace_closest_host': ([P, P, U32, P, P], ctypes.c_int),
        'vs_trace_any_device': ([P, P, U32, P, P], ctypes.c_int),
        'vs_trace_any_host': ([P, P, U32, P], ctypes.c_int),
        'vs_rgb_to_spectrum': ([P, ctypes.c_char_p, P, ctypes.c_int, P], ctypes.c_int),
        'vs_launch_count': ([], ctypes.c_uint64),
        'vs_sampler_stream': ([P, ctypes.c_int, U32, P, U32, U32, P], ctypes.c_int),
        'vs_render_stats': ([P, U32, U32, P], ctypes.c_int),
        'vs_timing_enable': ([P, ctypes.c_int], ctypes.c_int),
        'vs_timing_read': ([P, P, P, P], ctypes.c_int),
        'vs_render_noalloc': ([P, U32, U32, P, P], ctypes.c_int),
        'vs_render_schedule_set': ([P, ctypes.c_int], ctypes.c_int),
        'vs_cache_download': ([P, ctypes.c_int, P, ctypes.c_size_t], ctypes.c_int),
        'vs_albedo_luts': ([ctypes.c_int, ctypes.c_char_p, P, ctypes.c_size_t], ctypes.c_int),
        'vs_albedo_luts_gpu': ([P, U32, P, ctypes.c_size_t], ctypes.c_int),
        'vs_restir_frame': ([P, U32, U32, P], ctypes.c_int),
        'vs_restir_reset': ([P], ctypes.c_int),
        'vs_restir_params': ([P, U32, P, ctypes.c_size_t], ctypes.c_int),
        'vs_restir_download': ([P, ctypes.c_int, P, ctypes.c_size_t], ctypes.c_int),
        'vs_denoiser_enable': ([P, ctypes.c_int], ctypes.c_int),
        'vs_denoiser_params': ([P, P, ctypes.c_size_t], ctypes.c_int),
        'vs_server_create': ([P, ctypes.c_uint64, U32, ctypes.c_uint64, ctypes.POINTER(P)], ctypes.c_int),
        'vs_server_destroy': ([P], None),
        'vs_server_add_scene': ([P, P, ctypes.POINTER(U32)], ctypes.c_int),
        'vs_server_submit': ([P, ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        'vs_server_poll': ([P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
        'vs_server_result': ([P, ctypes.c_uint64, P, ctypes.c_size_t, ctypes.c_double], ctypes.c_int),
        'vs_server_stats_get': ([P, ctypes.POINTER(ServerStats)], ctypes.c_int),
        'vs_server_last_error': ([P], ctypes.c_char_p),
        'vs_cache_create': ([P, ctypes.c_uint64, ctypes.POINTER(P)], ctypes.c_int),
        'vs_cache_destroy': ([P], None),
        'vs_cache_get_weights': ([P, P, ctypes.c_size_t], ctypes.c_int),
        'vs_cache_set_weights': ([P, P, ctypes.c_size_t], ctypes.c_int),
        'vs_cache_set_optimizer': ([P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float], ctypes.c_int),
        'vs_cache_infer': ([P, P, U32, P, P], ctypes.c_int),
        'vs_cache_train': ([P, P, P, U32, ctypes.c_int, P], ctypes.c_int),
        'vs_cache_gradient': ([P, P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        'vs_render_cached': ([P, P, U32, U32, U32, ctypes.c_int, P], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()

# Symbols declared in include/vision_b200.h (checked by the CPU tests).
ABI_SYMBOLS = sorted(['vs_version', 'vs_context_create', 'vs_context_destroy', 'vs_last_error', 'vs_scene_load_json',
                      'vs_scene_destroy', 'vs_scene_build_accel', 'vs_set_resolution', 'vs_camera_set',
                      'vs_scene_info_get', 'vs_scene_export_size', 'vs_scene_export', 'vs_render', 'vs_synchronize',
                      'vs_film_download', 'vs_trace_closest_device', 'vs_trace_closest_host', 'vs_trace_any_device',
                      'vs_trace_any_host', 'vs_rgb_to_spectrum', 'vs_launch_count', 'vs_render_stats', 'vs_timing_enable',
                      'vs_timing_read', 'vs_render_noalloc', 'vs_albedo_luts', 'vs_albedo_luts_gpu', 'vs_restir_frame',
                      'vs_restir_reset', 'vs_restir_params', 'vs_restir_download', 'vs_server_create',
                      'vs_server_destroy', 'vs_server_add_scene', 'vs_server_submit', 'vs_server_poll',
                      'vs_server_result', 'vs_server_stats_get', 'vs_server_last_error', 'vs_cache_create',
                      'vs_cache_destroy', 'vs_cache_get_weights', 'vs_cache_set_weights', 'vs_cache_set_optimizer',
                      'vs_cache_infer', 'vs_cache_train', 'vs_cache_gradient', 'vs_render_cached',
                      'vs_render_schedule_set', 'vs_cache_download', 'vs_sampler_stream', 'vs_scene_add_instance',
                      'vs_scene_clear_geometries', 'vs_scene_invalidate', 'vs_denoiser_enable',
                      'vs_denoiser_params'])
CACHE_PARAMS = 16576
SCHEDULE_GRID = 0
# Buffers of the last cache-terminated frame (include/vision_b200.h VS_CACHE_*).
CACHE_QUERY_DTYPE = np.dtype([('t', '<f4', 4), ('lambda', '<f4', 4), ('pdf', '<f4', 4), ('l_valid', '<f4', 4)])
CACHE_TRAIN_DTYPE = np.dtype([('suffix_valid', '<f4', 4), ('t', '<f4', 4), ('lambda', '<f4', 4), ('pdf', '<f4', 4)])
CACHE_BUFFERS = dict(query_features=(0, np.dtype(('<u2', 64)), True), query_records=(1, CACHE_QUERY_DTYPE, True),
                     query_output=(2, np.dtype(('<f4', 4)), True), train_features=(3, np.dtype(('<u2', 64)), False),
                     train_records=(4, CACHE_TRAIN_DTYPE, False), suffix_features=(5, np.dtype(('<u2', 64)), False),
                     suffix_output=(6, np.dtype(('<f4', 4)), False), targets=(7, np.dtype(('<f4', 4)), False))
SCHEDULE_PERSISTENT = 1
SCHEDULE_WAVEFRONT = 2
SCHEDULE_WAVEFRONT_BINNED = 3

# Per-pixel ReSTIR records (vision_b200/csrc/vs_restir.h) as numpy dtypes.
HIT_DTYPE = np.dtype([('inst_id', '<u4'), ('prim_id', '<u4'), ('u', '<f4'), ('v', '<f4')])
RT_SURFACE_DTYPE = np.dtype([('hit', HIT_DTYPE), ('normal', '<f4', 3), ('depth', '<f4'), ('pos', '<f4', 3),
                             ('diffuse', '<f4'), ('is_replaced', '<u4'), ('flag', '<u4'), ('pad', '<u4', 2)])
DI_RESERVOIR_DTYPE = np.dtype([('weight_sum', '<f8'), ('C', '<f4'), ('W', '<f4'), ('light_index', '<u4'),
                               ('prim_id', '<u4'), ('bary', '<f4', 2), ('age', '<u4'), ('p_hat', '<f4'),
                               ('pos', '<f4', 3), ('pad', '<u4', 3)])
GI_RESERVOIR_DTYPE = np.dtype([('weight_sum', '<f8'), ('C', '<f4'), ('W', '<f4'), ('sp_pos', '<f4', 3),
                               ('sp_ng', '<f4', 3), ('Lo', '<f4', 3), ('age', '<f4'), ('pad', '<u4', 2)])
HIT_BSDF_DTYPE = np.dtype([('wi', '<f4', 3), ('f', '<f4', 3), ('pdf', '<f4'), ('pad', '<u4')])
RESTIR_PARAMS_BYTES = 448
# SVGF records: PixelGeometry and SVGFData (vs_restir.h SvgfGeom / SvgfData).
SVGF_GEOM_DTYPE = np.dtype([('normal', '<f4', 3), ('fwidth', '<f4'), ('p_film', '<f4', 2), ('depth_gradient', '<f4'),
                            ('linear_depth', '<f4')])
SVGF_DATA_DTYPE = np.dtype([('illumination', '<f4', 3), ('variance', '<f4'), ('history', '<f4'), ('moments', '<f4', 2),
                            ('pad', '<f4')])
SVGF_PARAMS_DTYPE = np.dtype([('N', '<u4'), ('alpha', '<f4'), ('moments_alpha', '<f4'), ('history_limit', '<u4'),
                              ('moments_radius', '<i4'), ('sigma_rt', '<f4'), ('sigma_normal', '<f4'),
                              ('reproject', '<u4'), ('filter_moments', '<u4'), ('pad', '<u4', 3)])
RESTIR = dict(di_radiance=(0, np.dtype(('<f4', 4))), gi_radiance=(1, np.dtype(('<f4', 4))),
              motion=(2, np.dtype(('<f4', 2))), surfaces=(3, RT_SURFACE_DTYPE), di_reservoirs=(4, DI_RESERVOIR_DTYPE),
              gi_reservoirs=(5, GI_RESERVOIR_DTYPE), hit_bsdf=(6, HIT_BSDF_DTYPE), gi_samples=(7, GI_RESERVOIR_DTYPE),
              denoised=(8, np.dtype(('<f4', 4))), gbuffer=(9, SVGF_GEOM_DTYPE),
              svgf_albedo=(10, np.dtype(('<f4', 4))), svgf_emission=(11, np.dtype(('<f4', 4))),
              svgf_data=(12, SVGF_DATA_DTYPE), svgf_motion=(13, np.dtype(('<f4', 2))),
              svgf_history=(14, np.dtype('<f4')))
assert SVGF_GEOM_DTYPE.itemsize == 32 and SVGF_DATA_DTYPE.itemsize == 32 and SVGF_PARAMS_DTYPE.itemsize == 48
assert RT_SURFACE_DTYPE.itemsize == 64 and DI_RESERVOIR_DTYPE.itemsize == 64 and GI_RESERVOIR_DTYPE.itemsize == 64


def launch_count():
    """Kernels launched by libvision_b200 since it was loaded."""
    return int(lib.vs_launch_count())


def sampler_stream(ctx, keys, draws, kind=0, seed=0):
    """Device sampler draws: keys is (count, 4) uint32 (px, py, sample, dim);
    returns (count, draws) float32 from the GPU sampler (kind 0 independent,
    1 PCG32 with stream `seed`)."""
    keys = np.ascontiguousarray(keys, np.uint32).reshape(-1, 4)
    out = np.zeros((keys.shape[0], draws), np.float32)
    ctx.check(lib.vs_sampler_stream(ctx.handle, kind, seed, _ptr(keys), keys.shape[0], draws, _ptr(out)),
              'sampler_stream')
    return out


LUT_FLOATS = 164864


def albedo_luts(regenerated=False):
    """Albedo tables of the compensated lobes: shipped (reference) or regenerated."""
    out = np.zeros(LUT_FLOATS, np.float32)
    rc = lib.vs_albedo_luts(1 if regenerated else 0, os.path.join(HERE, 'data', 'albedo_luts_regen.bin').encode(),
                            out.ctypes.data_as(ctypes.c_void_p), out.size)
    if rc != VS_OK:
        raise VisionError(rc, 'vs_albedo_luts failed')
    return out


def albedo_luts_gpu(ctx, strata=32):
    """Albedo tables regenerated on the context's GPU with strata^2 samples
    per cell (strata = 32: the estimator of albedo_luts(regenerated=True))."""
    out = np.zeros(LUT_FLOATS, np.float32)
    ctx.check(lib.vs_albedo_luts_gpu(ctx.handle, int(strata), out.ctypes.data_as(ctypes.c_void_p), out.size),
              'albedo_luts_gpu')
    return out


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class Context:
    """CUDA device context (device=-1: host only, for parsing and export)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib.vs_context_create(device, ctypes.byref(h))
        if rc != VS_OK:
            raise VisionError(rc, 'vs_context_create(%d) failed' % device)
        self.handle = h
        self.device = device

    def check(self, rc, what):
        if rc != VS_OK:
            msg = '%s: %s' % (what, lib.vs_last_error(self.handle).decode('utf-8', 'replace'))
            raise (UnsupportedError if rc == VS_E_UNSUPPORTED else VisionError)(rc, msg)

    def rgb_to_spectrum(self, rgb, mode=0):
        out = np.zeros(4, np.float32)
        self.check(lib.vs_rgb_to_spectrum(self.handle, TABLE_CACHE.encode(), _ptr(np.asarray(rgb, np.float32)),
                                          mode, _ptr(out)), 'rgb_to_spectrum')
        return out

    def close(self):
        if self.handle:
            lib.vs_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """A loaded vision_scene.json.  Mirrors Pipeline::prepare/render and the SDK
    calls build_accel / update_camera / render / download_radiance."""

    def __init__(self, ctx, scene, base_dir='.'):
        os.makedirs(os.path.dirname(TABLE_CACHE), exist_ok=True)
        self.ctx = ctx
        text = scene if isinstance(scene, str) else json.dumps(scene)
        data = text.encode()
        h = ctypes.c_void_p()
        ctx.check(lib.vs_scene_load_json(ctx.handle, data, len(data), base_dir.encode(), TABLE_CACHE.encode(),
                                         ctypes.byref(h)), 'load scene')
        self.handle = h
        self.frames = 0

    def build_accel(self):
        self.ctx.check(lib.vs_scene_build_accel(self.handle), 'build_accel')
        return self

    def info(self):
        i = SceneInfo()
        self.ctx.check(lib.vs_scene_info_get(self.handle, ctypes.byref(i)), 'scene info')
        return {n: getattr(i, n) for n, _ in SceneInfo._fields_}

    def export(self, what, dtype=np.uint8):
        key = EXPORT[what]
        n = ctypes.c_size_t()
        self.ctx.check(lib.vs_scene_export_size(self.handle, key, ctypes.byref(n)), 'export size')
        buf = np.zeros(max(n.value, 1), np.uint8)
        self.ctx.check(lib.vs_scene_export(self.handle, key, _ptr(buf), n.value), 'export')
        return buf[:n.value].view(dtype)

    def add_instance(self, positions, triangles, normals=None, uvs=None, o2w=None, material=None):
        """VisionRenderer::add_instance: positions (n, 3), triangles (m, 3),
        optional normals (n, 3) and uvs (n, 2), o2w a row-major 4x4 (stored
        column-major for the C ABI), material a name, a dict (material node)
        or None.  Returns the instance id; build_accel must follow."""
        p = np.asarray(positions, np.float32).reshape(-1, 3)
        v = np.zeros((p.shape[0], 10), np.float32)
        v[:, 0:3] = p
        if normals is not None:
            v[:, 3:6] = np.asarray(normals, np.float32).reshape(-1, 3)
        if uvs is not None:
            v[:, 6:8] = np.asarray(uvs, np.float32).reshape(-1, 2)
        t = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
        m = None if o2w is None else np.ascontiguousarray(np.asarray(o2w, np.float32).T)
        mat = material if material is None or isinstance(material, str) else json.dumps(material)
        inst = ctypes.c_uint32()
        self.ctx.check(lib.vs_scene_add_instance(self.handle, _ptr(v), p.shape[0], _ptr(t), t.shape[0], _ptr(m),
                                                 mat.encode() if mat else None, ctypes.byref(inst)), 'add_instance')
        self.frames = 0
        return inst.value

    def clear_geometries(self):
        self.ctx.check(lib.vs_scene_clear_geometries(self.handle), 'clear_geometries')
        self.frames = 0

    def invalidate(self):
        self.ctx.check(lib.vs_scene_invalidate(self.handle), 'invalidate')
        self.frames = 0

    def set_resolution(self, w, h):
        self.ctx.check(lib.vs_set_resolution(self.handle, w, h), 'set_resolution')
        self.frames = 0

    def render(self, frame_begin, frame_count, fp64=False, stream=None):
        self.ctx.check(lib.vs_render(self.handle, frame_begin, frame_count, FILM_FP64 if fp64 else FILM_FP32,
                                     ctypes.c_void_p(stream) if stream else None), 'render')
        self.frames = frame_begin + frame_count

    def synchronize(self):
        self.ctx.check(lib.vs_synchronize(self.handle), 'synchronize')

    def film(self, which=FILM_LINEAR):
        i = self.info()
        npix = i['width'] * i['height']
        if which in (FILM_SUM64, FILM_SUMSQ64):
            out = np.zeros((i['height'], i['width'], 4), np.float64)
        elif which == FILM_RGBA8:
            out = np.zeros((i['height'], i['width'], 4), np.uint8)
        else:
            out = np.zeros((i['height'], i['width'], 4), np.float32)
        self.ctx.check(lib.vs_film_download(self.handle, _ptr(out), out.nbytes, which), 'film download')
        return out

    def trace_closest(self, rays):
        """rays: (n, 8) float32 host array -> (hits (n, 4) uint32 [inst, prim, u bits, v bits], t (n,))."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        hits = np.zeros((n, 4), np.uint32)
        t = np.zeros(n, np.float32)
        self.ctx.check(lib.vs_trace_closest_host(self.handle, _ptr(rays), n, _ptr(hits), _ptr(t)), 'trace_closest')
        return hits, t

    def trace_any(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint32)
        self.ctx.check(lib.vs_trace_any_host(self.handle, _ptr(rays), rays.shape[0], _ptr(occ)), 'trace_any')
        return occ

    def trace_closest_device(self, rays_ptr, n, hits_ptr, t_ptr, stream=None):
        self.ctx.check(lib.vs_trace_closest_device(self.handle, ctypes.c_void_p(rays_ptr), n, ctypes.c_void_p(hits_ptr),
                                                   ctypes.c_void_p(t_ptr), ctypes.c_void_p(stream) if stream else None),
                       'trace_closest_device')

    def set_schedule(self, schedule):
        """Path scheduling of render(): 'wavefront' (bounces as separate
        kernels over path state in device memory, the default), 'persistent'
        (regenerating resident wave), 'grid' (one path per thread) or
        'wavefront_binned' (the wavefront with rays grouped by direction octant
        and origin cell before each traversal pass)."""
        code = {'grid': SCHEDULE_GRID, 'persistent': SCHEDULE_PERSISTENT, 'wavefront': SCHEDULE_WAVEFRONT,
                'wavefront_binned': SCHEDULE_WAVEFRONT_BINNED}[schedule]
        self.ctx.check(lib.vs_render_schedule_set(self.handle, code), 'render_schedule_set')

    def timing_enable(self, on=True):
        self.ctx.check(lib.vs_timing_enable(self.handle, 1 if on else 0), 'timing_enable')

    def timing_read(self):
        """(megakernel ms, film ms, megakernel launches) since timing_enable."""
        r = ctypes.c_double()
        f = ctypes.c_double()
        n = ctypes.c_uint32()
        self.ctx.check(lib.vs_timing_read(self.handle, ctypes.byref(r), ctypes.byref(f), ctypes.byref(n)), 'timing_read')
        return r.value, f.value, n.value

    def set_camera(self, c2w, fov_y_deg):
        """Camera-to-world 4x4 (row-major numpy matrix; passed column-major) and fov."""
        m = np.ascontiguousarray(np.asarray(c2w, np.float32).T)
        self.ctx.check(lib.vs_camera_set(self.handle, _ptr(m), float(fov_y_deg)), 'camera_set')
        self.frames = 0

    def restir_frame(self, frame_index, film_index=None, stream=None):
        """One real-time ReSTIR frame (scene integrator "rt"); the film gets the
        frame as sample `film_index` of its running mean (default: next)."""
        fi = self.frames if film_index is None else film_index
        self.ctx.check(lib.vs_restir_frame(self.handle, frame_index, fi, ctypes.c_void_p(stream) if stream else None),
                       'restir_frame')
        self.frames = fi + 1

    def restir_reset(self):
        self.ctx.check(lib.vs_restir_reset(self.handle), 'restir_reset')

    def restir_params(self, frame_index):
        """Parameter block (bytes) of a vs_restir_frame call made now with this frame index."""
        out = np.zeros(RESTIR_PARAMS_BYTES, np.uint8)
        self.ctx.check(lib.vs_restir_params(self.handle, frame_index, _ptr(out), out.nbytes), 'restir_params')
        return out

    def denoiser_enable(self, on=True):
        """SVGF after every restir_frame (read with restir_buffer('denoised'))."""
        self.ctx.check(lib.vs_denoiser_enable(self.handle, 1 if on else 0), 'denoiser_enable')

    def denoiser_params(self):
        """The SVGF settings block (SVGF_PARAMS_DTYPE)."""
        out = np.zeros(1, SVGF_PARAMS_DTYPE)
        self.ctx.check(lib.vs_denoiser_params(self.handle, _ptr(out), out.nbytes), 'denoiser_params')
        return out[0]

    def restir_buffer(self, which):
        key, dt = RESTIR[which]
        i = self.info()
        out = np.zeros(i['width'] * i['height'], dt)
        self.ctx.check(lib.vs_restir_download(self.handle, key, _ptr(out), out.nbytes), 'restir_download')
        return out.reshape((i['height'], i['width']) + out.shape[1:])

    def render_cached(self, cache, frame_begin, frame_count, train_samples=65536, fp64=False, stream=None):
        """Cache-terminated frames; the cache trains on train_samples paths per frame."""
        self.ctx.check(lib.vs_render_cached(self.handle, cache.handle, frame_begin, frame_count, train_samples,
                                            FILM_FP64 if fp64 else FILM_FP32,
                                            ctypes.c_void_p(stream) if stream else None), 'render_cached')
        self.frames = frame_begin + frame_count
        if frame_count:
            i = self.info()
            self._cache_train = min(train_samples, i['width'] * i['height'])

    def cache_buffer(self, which):
        """A buffer of the last cache-terminated frame (CACHE_BUFFERS key):
        per-pixel arrays (height, width, ...) or per training sample (n, ...)."""
        key, dt, per_pixel = CACHE_BUFFERS[which]
        i = self.info()
        n = i['width'] * i['height'] if per_pixel else getattr(self, '_cache_train', 0)
        out = np.zeros(n, dt)
        self.ctx.check(lib.vs_cache_download(self.handle, key, _ptr(out), out.nbytes), 'cache_download')
        return out.reshape((i['height'], i['width']) + out.shape[1:]) if per_pixel else out

    def render_stats(self, frame_begin, frame_count):
        """Traversal counters of an instrumented render: (segments, nodes, tris)."""
        out = np.zeros(3, np.uint64)
        self.ctx.check(lib.vs_render_stats(self.handle, frame_begin, frame_count, _ptr(out)), 'render_stats')
        return tuple(int(x) for x in out)

    def close(self):
        if self.handle:
            lib.vs_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Render-job server (vs_server_*): continuous batching of path-tracing
    jobs over resident scenes; jobs on a real-time (rt) scene run ReSTIR
    frames with the scene's reservoirs resident from job to job."""

    def __init__(self, ctx, hbm_budget=150 << 30, max_jobs=64, paths_per_batch=1 << 23):
        h = ctypes.c_void_p()
        ctx.check(lib.vs_server_create(ctx.handle, hbm_budget, max_jobs, paths_per_batch, ctypes.byref(h)),
                  'server_create')
        self.ctx = ctx
        self.handle = h
        self.scenes = []
        self.sizes = {}

    def check(self, rc, what):
        if rc != VS_OK:
            msg = '%s: %s' % (what, lib.vs_server_last_error(self.handle).decode())
            raise (UnsupportedError if rc == VS_E_UNSUPPORTED else VisionError)(rc, msg)

    def add_scene(self, scene):
        sid = ctypes.c_uint32()
        self.check(lib.vs_server_add_scene(self.handle, scene.handle, ctypes.byref(sid)), 'add_scene')
        self.scenes.append(scene)  # the scene must outlive its use by the server
        return sid.value

    def submit(self, scene_id, width, height, spp, frame_begin=0, c2w=None, fov_y=0.0):
        d = JobDesc()
        d.scene, d.width, d.height, d.spp, d.frame_begin = scene_id, width, height, spp, frame_begin
        d.fov_y_deg = fov_y
        if c2w is not None:
            d.use_c2w = 1
            m = np.asarray(c2w, np.float32).T.reshape(-1)
            for i in range(16):
                d.c2w[i] = float(m[i])
        jid = ctypes.c_uint64()
        self.check(lib.vs_server_submit(self.handle, ctypes.byref(d), ctypes.byref(jid)), 'submit')
        self.sizes[jid.value] = (height, width)
        return jid.value

    def poll(self, job):
        done = ctypes.c_int()
        self.check(lib.vs_server_poll(self.handle, job, ctypes.byref(done)), 'poll')
        return bool(done.value)

    def result(self, job, timeout=-1.0):
        h, w = self.sizes.pop(job)
        out = np.zeros((h, w, 4), np.float32)
        self.check(lib.vs_server_result(self.handle, job, _ptr(out), out.nbytes, timeout), 'result')
        return out

    def stats(self):
        s = ServerStats()
        self.check(lib.vs_server_stats_get(self.handle, ctypes.byref(s)), 'stats')
        return {n: getattr(s, n) for n, _ in ServerStats._fields_}

    def close(self):
        if self.handle:
            lib.vs_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RadianceCache:
    """Radiance-cache MLP on the tensor cores (vs_cache_*).  Feature and
    output buffers are device pointers (e.g. torch tensors' data_ptr())."""

    def __init__(self, ctx, seed=1):
        h = ctypes.c_void_p()
        ctx.check(lib.vs_cache_create(ctx.handle, seed, ctypes.byref(h)), 'cache_create')
        self.ctx = ctx
        self.handle = h

    def weights(self):
        w = np.zeros(CACHE_PARAMS, np.float32)
        self.ctx.check(lib.vs_cache_get_weights(self.handle, _ptr(w), w.size), 'cache weights')
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self.ctx.check(lib.vs_cache_set_weights(self.handle, _ptr(w), w.size), 'cache set weights')

    def set_optimizer(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.ctx.check(lib.vs_cache_set_optimizer(self.handle, lr, beta1, beta2, eps), 'cache optimizer')

    def infer(self, feat_ptr, n, out_ptr, stream=None):
        self.ctx.check(lib.vs_cache_infer(self.handle, ctypes.c_void_p(feat_ptr), n, ctypes.c_void_p(out_ptr),
                                          ctypes.c_void_p(stream) if stream else None), 'cache infer')

    def train(self, feat_ptr, target_ptr, n, update=True, stream=None):
        self.ctx.check(lib.vs_cache_train(self.handle, ctypes.c_void_p(feat_ptr), ctypes.c_void_p(target_ptr), n,
                                          1 if update else 0, ctypes.c_void_p(stream) if stream else None),
                       'cache train')

    def gradient(self):
        g = np.zeros(CACHE_PARAMS, np.float32)
        loss = ctypes.c_double()
        self.ctx.check(lib.vs_cache_gradient(self.handle, _ptr(g), g.size, ctypes.byref(loss)), 'cache gradient')
        return g, loss.value

    def close(self):
        if self.handle:
            lib.vs_cache_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
