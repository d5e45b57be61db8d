"""Builds libvision_b200.so in-tree with nvcc for sm_100a.

usage: python vision_b200/build.py [--force] [-v]

Objects go to vision_b200/_build/; the shared library lands next to this file
so that it travels with the package.  Rebuilds only when a source or header is
newer than the library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libvision_b200.so')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')

SOURCES = ['kernels.cu', 'restir.cu', 'server.cu', 'mlp.cu', 'cache_render.cu', 'capi.cu', 'noalloc.cu', 'scene_load.cpp', 'bvh8.cpp', 'rgb2spec.cpp', 'luts.cpp']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC,-ffp-contract=off,-pthread',
          '-I', CSRC, '-I', INCLUDE]


def nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def _newest_input():
    t = 0.0
    for root, _, files in os.walk(CSRC):
        for f in files:
            t = max(t, os.path.getmtime(os.path.join(root, f)))
    t = max(t, os.path.getmtime(os.path.join(INCLUDE, 'vision_b200.h')))
    return t


def up_to_date():
    return os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input()


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
        cmd = [nvcc()] + ARCH + COMMON + ['-c', os.path.join(CSRC, src), '-o', obj]
        if src.endswith('.cu'):
            cmd += ['-Xptxas', '-v'] if verbose else []
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + '.tmp'
    subprocess.run([nvcc()] + ARCH + ['-shared', '-o', tmp] + objs + ['-lcudart', '-lpthread'], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
