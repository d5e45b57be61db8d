"""Builds libvision_b200.so in-tree with nvcc for sm_100a.

usage: python vision_b200/build.py [--force] [-v]

Objects go to vision_b200/_build/; the shared library lands next to this file
so that it travels with the package.  Each object and the library carry a
digest of their sources, headers and flags (`.stamp` files); only objects
whose digest changed are recompiled, in parallel.
"""
import concurrent.futures
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libvision_b200.so')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')

SOURCES = ['kernels.cu', 'wavefront.cu', 'restir.cu', 'restir_diffuse.cu', 'svgf.cu', 'server.cu', 'mlp.cu', 'cache_render.cu', 'capi.cu', 'noalloc.cu', 'scene_load.cpp', 'image_io.cpp', 'bvh8.cpp', 'rgb2spec.cpp', 'luts.cpp', 'lut_gen.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC,-ffp-contract=off,-pthread',
          '-I', CSRC, '-I', INCLUDE]
# Per-source device flags.  svgf.cu: no multiply-add contraction, as in the
# host oracle; its edge-stopping weights (exp of depth and luminance
# differences over small sigmas) magnify one-ulp differences in the G-buffer.
SOURCE_FLAGS = {'svgf.cu': ['--fmad=false']}


def nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def _digest(paths, extra):
    h = hashlib.sha256()
    for p in paths:
        h.update(p.encode())
        with open(p, 'rb') as f:
            h.update(f.read())
    h.update(' '.join(extra).encode())
    return h.hexdigest()


def _headers():
    hs = [os.path.join(INCLUDE, 'vision_b200.h')]
    for root, _, files in os.walk(CSRC):
        for f in sorted(files):
            if not f.endswith(('.cu', '.cpp')):
                hs.append(os.path.join(root, f))
    return sorted(hs)


def _source_digest(src):
    return _digest([os.path.join(CSRC, src)] + _headers(), ARCH + COMMON + SOURCE_FLAGS.get(src, []))


def _library_digest():
    flags = [f for src in SOURCES for f in SOURCE_FLAGS.get(src, [])]
    return _digest([os.path.join(CSRC, s) for s in SOURCES] + _headers(), ARCH + COMMON + SOURCES + flags)


def _stamp_ok(path, digest):
    stamp = path + '.stamp'
    return os.path.exists(path) and os.path.exists(stamp) and open(stamp).read().strip() == digest


def up_to_date():
    """True when the library was built from exactly the current sources and
    flags (content digest, so copies with fresh file times stay valid)."""
    return _stamp_ok(LIB, _library_digest())


def build(force=False, verbose=False):
    # The digest of the sources as they are now: a source edited while the
    # build runs leaves the library stale, not stamped as current.
    lib_digest = _library_digest()
    if not force and _stamp_ok(LIB, lib_digest):
        return LIB
    os.makedirs(BUILD, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
        digest = _source_digest(src)
        if not force and _stamp_ok(obj, digest):
            return obj
        cmd = [nvcc()] + ARCH + COMMON + SOURCE_FLAGS.get(src, []) + ['-c', os.path.join(CSRC, src), '-o', obj]
        if src.endswith('.cu') and verbose:
            cmd += ['-Xptxas', '-v']
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
        with open(obj + '.stamp', 'w') as f:
            f.write(digest)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB + '.tmp'
    subprocess.run([nvcc()] + ARCH + ['-shared', '-o', tmp] + objs + ['-lcudart', '-lpthread'], check=True)
    os.replace(tmp, LIB)
    with open(LIB + '.stamp', 'w') as f:
        f.write(lib_digest)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
