"""ORACLE — test infrastructure only.

ctypes bridge to the CPU restatement in oracle/oracle.cpp.  Imported only by
tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, always
as the checker and never as the thing measured or shipped.  The parity status
of the oracle (what pins it, what is unpinned) is stated in oracle.cpp's
header.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_build', 'liboracle.so')


FMA_LIB_PATH = os.path.join(HERE, '_build', 'liboracle_fma.so')


def build():
    srcs = [os.path.join(HERE, f) for f in ('oracle.cpp', 'restir.inc', 'Makefile')]
    newest = max(os.path.getmtime(s) for s in srcs)
    if all(os.path.exists(p) and os.path.getmtime(p) >= newest for p in (LIB_PATH, FMA_LIB_PATH)):
        return LIB_PATH
    subprocess.run(['make', '-s', '-C', HERE], check=True)
    return LIB_PATH


class OracleSceneStruct(ctypes.Structure):
    _fields_ = [('pos', ctypes.c_void_p), ('nrm', ctypes.c_void_p), ('uv', ctypes.c_void_p), ('idx', ctypes.c_void_p),
                ('prim_inst', ctypes.c_void_p), ('vertex_count', ctypes.c_uint32), ('prim_count', ctypes.c_uint32),
                ('instances', ctypes.c_void_p), ('instance_count', ctypes.c_uint32),
                ('materials', ctypes.c_void_p), ('material_count', ctypes.c_uint32),
                ('lights', ctypes.c_void_p), ('light_count', ctypes.c_uint32),
                ('prim_alias', ctypes.c_void_p), ('prim_pmf', ctypes.c_void_p),
                ('light_alias', ctypes.c_void_p), ('light_pmf', ctypes.c_void_p),
                ('camera', ctypes.c_void_p), ('integrator', ctypes.c_void_p), ('spd', ctypes.c_void_p),
                ('env', ctypes.c_void_p), ('env_tex', ctypes.c_void_p), ('env_marginal', ctypes.c_void_p),
                ('env_marginal_func', ctypes.c_void_p), ('env_cond', ctypes.c_void_p),
                ('env_cond_func', ctypes.c_void_p), ('rgb2spec', ctypes.c_void_p),
                ('two_level', ctypes.c_uint32), ('mesh_count', ctypes.c_uint32), ('mesh_pos', ctypes.c_void_p),
                ('mesh_idx', ctypes.c_void_p), ('meshes', ctypes.c_void_p), ('inst_mesh', ctypes.c_void_p),
                ('inst_w2o', ctypes.c_void_p), ('tex_texels', ctypes.c_void_p), ('textures', ctypes.c_void_p),
                ('texture_count', ctypes.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        U = ctypes.c_uint32
        L.oracle_open.argtypes = [P]
        L.oracle_open.restype = P
        L.oracle_close.argtypes = [P]
        L.oracle_trace_closest.argtypes = [P, P, U, P, P]
        L.oracle_trace_any.argtypes = [P, P, U, P]
        L.oracle_paths.argtypes = [P, P, U, U, U, U, P]
        L.oracle_render.argtypes = [P, U, U, U, P, P]
        L.oracle_sampler_stream.argtypes = [U, U, U, U, U, U, U, P]
        L.oracle_tea.argtypes = [U, U]
        L.oracle_tea.restype = U
        L.oracle_wavelengths.argtypes = [U, ctypes.c_float, P, P]
        L.oracle_linear_srgb.argtypes = [U, P, P, P, P]
        L.oracle_cie_y_integral.restype = ctypes.c_float
        L.oracle_spd_eval.argtypes = [P, ctypes.c_int, ctypes.c_float]
        L.oracle_spd_eval.restype = ctypes.c_float
        L.oracle_rt_open.argtypes = [P, U, U]
        L.oracle_rt_open.restype = P
        L.oracle_rt_close.argtypes = [P]
        L.oracle_rt_frame.argtypes = [P, P, P, U, U]
        L.oracle_rt_buffer.argtypes = [P, ctypes.c_int, P, ctypes.c_size_t]
        L.oracle_rt_svgf.argtypes = [P, P, P, P, P, U]
        _lib = L
    return _lib


_fma_lib = None


def fma_lib():
    """The oracle compiled with FMA contraction (same source, different
    rounding): renders through it differ from the oracle's by rounding only."""
    global _fma_lib
    if _fma_lib is None:
        build()
        L = ctypes.CDLL(FMA_LIB_PATH)
        for fn in ('oracle_open', 'oracle_close', 'oracle_render'):
            getattr(L, fn).argtypes = getattr(lib(), fn).argtypes
            getattr(L, fn).restype = getattr(lib(), fn).restype
        _fma_lib = L
    return _fma_lib


def render_fma(oscene, frame_begin, frame_count, threads=None):
    """FP64 film sums of an OracleScene rendered by the FMA-contracted oracle."""
    L = fma_lib()
    h = ctypes.c_void_p(L.oracle_open(ctypes.byref(oscene.s)))
    film = np.zeros((oscene.height, oscene.width, 4), np.float32)
    f64 = np.zeros((oscene.height, oscene.width, 4), np.float64)
    try:
        L.oracle_render(h, frame_begin, frame_count, threads or os.cpu_count(), _p(film), _p(f64))
    finally:
        L.oracle_close(h)
    return f64


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


SCENE_KEYS = ['pos', 'nrm', 'uv', 'idx', 'prim_inst', 'instances', 'materials', 'lights', 'prim_alias', 'prim_pmf',
              'light_alias', 'light_pmf', 'camera', 'integrator', 'spd']
ENV_KEYS = ['env', 'env_tex', 'env_marginal', 'env_marginal_func', 'env_cond', 'env_cond_func', 'rgb2spec']
INSTANCE_KEYS = ['mesh_pos', 'mesh_idx', 'meshes', 'inst_mesh', 'inst_w2o']
TEXTURE_KEYS = ['tex_texels', 'textures']


class OracleScene:
    """A flat scene held alive for the oracle: either the arrays exported by a
    vision_b200.Scene (OracleScene(scene): the oracle traces exactly the
    library's triangles and records), or the oracle's own ingestion of the
    scene document (OracleScene.from_json(doc), oracle/scene.py), which does
    not load the library at all."""

    def __init__(self, scene=None, arrays=None, info=None):
        if scene is not None:
            env = scene.export('env')
            info = scene.info()
            textures = scene.export('textures')
            keys = SCENE_KEYS + (ENV_KEYS if env.size else []) + (INSTANCE_KEYS if info.get('two_level') else [])
            keys += TEXTURE_KEYS + ['rgb2spec'] if textures.size else []
            arrays = {k: scene.export(k) for k in dict.fromkeys(keys)}
        has_env = 'env' in arrays and arrays['env'].size > 0
        two_level = bool(info.get('two_level')) and 'mesh_pos' in arrays
        has_tex = 'textures' in arrays and arrays['textures'].size > 0
        self.arr = {}
        keys = SCENE_KEYS + (ENV_KEYS if has_env else []) + (INSTANCE_KEYS if two_level else [])
        keys += TEXTURE_KEYS + ['rgb2spec'] if has_tex else []
        for k in dict.fromkeys(keys):
            a = np.ascontiguousarray(arrays[k])
            if a.size == 0:
                a = np.zeros(16, np.uint8)
            self.arr[k] = a
        self.info = info
        self.width, self.height = info['width'], info['height']
        a = self.arr
        self.s = OracleSceneStruct(_p(a['pos']), _p(a['nrm']), _p(a['uv']), _p(a['idx']), _p(a['prim_inst']),
                                   info['vertex_count'], info['prim_count'], _p(a['instances']), info['instance_count'],
                                   _p(a['materials']), info['material_count'], _p(a['lights']), info['light_count'],
                                   _p(a['prim_alias']), _p(a['prim_pmf']), _p(a['light_alias']), _p(a['light_pmf']),
                                   _p(a['camera']), _p(a['integrator']), _p(a['spd']),
                                   *([_p(a[k]) for k in ENV_KEYS[:-1]] if has_env else [None] * 6),
                                   _p(a['rgb2spec']) if has_env or has_tex else None,
                                   1 if two_level else 0, int(info.get('mesh_count', 0)) if two_level else 0,
                                   *([_p(a[k]) for k in INSTANCE_KEYS] if two_level else [None] * 5),
                                   *([_p(a[k]) for k in TEXTURE_KEYS] if has_tex else [None] * 2),
                                   a['textures'].view(np.uint8).size // 16 if has_tex else 0)
        self.h = ctypes.c_void_p(lib().oracle_open(ctypes.byref(self.s)))

    @classmethod
    def from_json(cls, doc, base_dir='.'):
        from oracle import scene as oscene
        arrays, info = oscene.build(doc, base_dir)
        return cls(arrays=arrays, info=info)

    def __del__(self):
        try:
            if self.h:
                lib().oracle_close(self.h)
                self.h = None
        except Exception:
            pass

    def trace_closest(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        hits = np.zeros((n, 4), np.uint32)
        t = np.zeros(n, np.float32)
        lib().oracle_trace_closest(self.h, _p(rays), n, _p(hits), _p(t))
        return hits, t

    def trace_any(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint32)
        lib().oracle_trace_any(self.h, _p(rays), rays.shape[0], _p(occ))
        return occ

    def render(self, frame_begin, frame_count, threads=None, fp64=False):
        threads = threads or os.cpu_count()
        film = np.zeros((self.height, self.width, 4), np.float32)
        f64 = np.zeros((self.height, self.width, 4), np.float64) if fp64 else None
        lib().oracle_render(self.h, frame_begin, frame_count, threads, _p(film),
                            _p(f64) if fp64 else None)
        return (film, f64) if fp64 else film

    def paths(self, pixels, frame_begin, frame_count, threads=None):
        pixels = np.ascontiguousarray(pixels, np.uint32)
        out = np.zeros((frame_count, pixels.size, 3), np.float32)
        lib().oracle_paths(self.h, _p(pixels), pixels.size, frame_begin, frame_count,
                           threads or os.cpu_count(), _p(out))
        return out


class OracleRestir:
    """CPU restatement of the real-time ReSTIR frame over an OracleScene."""

    BUFFERS = dict(di_radiance=0, gi_radiance=1, motion=2, surfaces=3, di_reservoirs=4, gi_reservoirs=5,
                   hit_bsdf=6, gi_samples=7, film=8, denoised=9, gbuffer=10, svgf_albedo=11, svgf_emission=12,
                   svgf_data=13, svgf_motion=14, svgf_history=15)

    def __init__(self, oscene, width, height):
        self.oscene = oscene
        self.width, self.height = width, height
        self.h = ctypes.c_void_p(lib().oracle_rt_open(oscene.h, width, height))

    def frame(self, camera, params, film_index, threads=None):
        camera = np.ascontiguousarray(camera).view(np.uint8)
        params = np.ascontiguousarray(params).view(np.uint8)
        assert camera.nbytes == 128 and params.nbytes == 448
        rc = lib().oracle_rt_frame(self.h, _p(camera), _p(params), film_index, threads or os.cpu_count())
        if rc != 0:
            raise ValueError('oracle_rt_frame rejected the parameters')

    def svgf(self, camera, params, svgf_params, radiance, threads=None):
        """SVGF over a film (height x width x 4 float32) with the frame's camera
        and parameter blocks and the 48-byte SVGF settings."""
        camera = np.ascontiguousarray(camera).view(np.uint8)
        params = np.ascontiguousarray(params).view(np.uint8)
        svgf_params = np.ascontiguousarray(svgf_params).view(np.uint8)
        radiance = np.ascontiguousarray(radiance, np.float32)
        assert camera.nbytes == 128 and params.nbytes == 448 and svgf_params.nbytes == 48
        assert radiance.size == 4 * self.width * self.height
        rc = lib().oracle_rt_svgf(self.h, _p(camera), _p(params), _p(svgf_params), _p(radiance),
                                  threads or os.cpu_count())
        if rc != 0:
            raise ValueError('oracle_rt_svgf rejected the parameters')

    def buffer(self, which, dtype):
        out = np.zeros(self.width * self.height, dtype)
        rc = lib().oracle_rt_buffer(self.h, self.BUFFERS[which], _p(out), out.nbytes)
        if rc != 0:
            raise ValueError('oracle_rt_buffer(%s) failed: %d' % (which, rc))
        return out.reshape((self.height, self.width) + out.shape[1:])

    def __del__(self):
        try:
            if self.h:
                lib().oracle_rt_close(self.h)
                self.h = None
        except Exception:
            pass


def sampler_stream(px, py, sample, dim, n, kind=0, seed=0):
    out = np.zeros(n, np.float32)
    lib().oracle_sampler_stream(px, py, sample, dim, kind, seed, n, _p(out))
    return out


def tea(a, b):
    return lib().oracle_tea(a, b)


def wavelengths(n, u):
    lam = np.zeros(n, np.float32)
    pdf = np.zeros(n, np.float32)
    lib().oracle_wavelengths(n, ctypes.c_float(u), _p(lam), _p(pdf))
    return lam, pdf


def linear_srgb(lam, pdf, s):
    lam = np.ascontiguousarray(lam, np.float32)
    pdf = np.ascontiguousarray(pdf, np.float32)
    s = np.ascontiguousarray(s, np.float32)
    rgb = np.zeros(3, np.float32)
    lib().oracle_linear_srgb(lam.size, _p(lam), _p(pdf), _p(s), _p(rgb))
    return rgb


def cie_y_integral():
    return lib().oracle_cie_y_integral()
