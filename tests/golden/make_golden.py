"""Generates the golden fixtures in tests/golden/ (run by hand; outputs are committed).

The reference ships no unit-test vectors for its path tracer; what it does ship
are its data tables and closed-form routines.  This script derives known
answers from those, in plain Python/numpy written directly from the cited
reference lines, independently of both the CUDA library and the C++ oracle:

  cie_5nm.json        the 94-entry 5 nm CIE X/Y/Z/D65 SPDs and the CIE Y
                      integral as the reference builds them
                      (src/base/color/spd.cpp:14-38,96-115) from its 1 nm
                      tables (src/base/color/cie.h:22-412)
  sampler.json        TEA(4 rounds) seeds and LCG streams of the independent
                      sampler (src/math/util.h:13-33,
                      src/render_core/samplers/independent.cpp:24-42)
  wavelengths.json    hero wavelength samples and pdfs
                      (src/render_core/spectra/hero.cpp:15-25,286-299)
  alias.json          Vose alias tables and PMFs
                      (src/render_core/warpers/alias.h:86-122,148-169)
  spd_eval.json       SPD::eval lookups with the reference's 471/n spacing
                      (src/base/color/spd.cpp:67-76)
  albedo_luts.json    the reference's precomputed lobe albedo tables
                      (src/base/scattering/precomputed_table.h): the full
                      32x32 PureReflectionLobe table and the Dielectric,
                      DielectricInv and Specular 32^3 tables on a 7^3 subgrid

usage: python tests/golden/make_golden.py <reference-root>
"""
import json
import os
import re
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
M32 = 0xffffffff


def tea(v0, v1):
    s0 = 0
    for _ in range(4):
        s0 = (s0 + 0x9e3779b9) & M32
        v0 = (v0 + ((((v1 << 4) & M32) + 0xa341316c) ^ ((v1 + s0) & M32) ^ ((v1 >> 5) + 0xc8013ea4))) & M32
        v1 = (v1 + ((((v0 << 4) & M32) + 0xad90777d) ^ ((v0 + s0) & M32) ^ ((v0 >> 5) + 0x7e95761e))) & M32
    return v0


def lcg_stream(state, n):
    out = []
    for _ in range(n):
        state = (1664525 * state + 1013904223) & M32
        out.append(float(np.float32(state & 0x00ffffff) * np.float32(1.0 / 16777216.0)))
    return out


def read_cie(ref):
    text = open(os.path.join(ref, 'src/base/color/cie.h')).read()
    tabs = {}
    for name in ('X', 'Y', 'Z', 'D65'):
        m = re.search(r'array<float, cie_sample_count>\s+%s\s*=\s*\{(.*?)\};' % name, text, re.S)
        body = re.sub(r'//[^\n]*', '', m.group(1))
        tabs[name] = np.array([float(x.rstrip('f')) for x in re.findall(r'[-+]?\d*\.\d+(?:[eE][-+]?\d+)?f?', body)],
                              np.float32)
    return tabs


def main():
    ref = sys.argv[1]
    tabs = read_cie(ref)
    # spd.cpp:31-38 downsample, :14-23 integral (float accumulation).
    down = {k: [float(v) for v in tabs[k][0:470:5][:94]] for k in tabs}
    s = np.float32(0.0)
    for i in range(94):
        s = np.float32(s + np.float32(0.5) * (tabs['Y'][5 * i] + tabs['Y'][5 * (i + 1)]))
    integral = float(np.float32(s * np.float32(5.0)))
    json.dump({'x': down['X'], 'y': down['Y'], 'z': down['Z'], 'd65': down['D65'], 'y_integral': integral},
              open(os.path.join(OUT, 'cie_5nm.json'), 'w'))

    rng = np.random.default_rng(7)
    cases = []
    for _ in range(32):
        px, py, smp = (int(v) for v in rng.integers(0, 4096, 3))
        dim = int(rng.choice([0, 0xffffffff]))
        seed = tea(tea(px, py), tea(smp, dim))
        cases.append({'px': px, 'py': py, 'sample': smp, 'dim': dim, 'seed': seed, 'stream': lcg_stream(seed, 12)})
    json.dump(cases, open(os.path.join(OUT, 'sampler.json'), 'w'))

    wl = []
    for n in (1, 3, 4):
        for u in [0.0, 0.1234, 0.5, 0.77, 0.999]:
            lam, pdf = [], []
            for i in range(n):
                off = np.float32(np.float32(i) * np.float32(np.float32(1.0) / np.float32(n)))
                up = np.float64(np.float32(np.float32(u) + off))
                up = up - np.floor(up)
                l = 538.0 - 138.888889 * np.arctanh(0.85691062 - 1.82750197 * up)
                lam.append(float(l))
                pdf.append(float(0.0039398042 / np.cosh(0.0072 * (l - 538.0)) ** 2))
            wl.append({'n': n, 'u': u, 'lambda': lam, 'pdf': pdf})
    json.dump(wl, open(os.path.join(OUT, 'wavelengths.json'), 'w'))

    al = []
    for weights in ([1.0], [1.0, 3.0], [0.5, 0.25, 0.25, 2.0], list(rng.random(17).astype(np.float32) + 0.01)):
        w = [float(np.float32(x)) for x in weights]
        n = len(w)
        total = sum(np.float64(x) for x in w)
        ratio = n / total
        table = []
        over, under = [], []
        for i, x in enumerate(w):
            p = float(np.float32(x * ratio))
            table.append([p, i])
            (over if p > 1.0 else under).append(i)
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
        integral = np.float32(total / n)
        pmf = [float(np.float32(x) / (integral * np.float32(n))) for x in w]
        al.append({'weights': w, 'table': table, 'pmf': pmf})
    json.dump(al, open(os.path.join(OUT, 'alias.json'), 'w'))

    ev = []
    for lam in (355.0, 360.0, 361.3, 400.0, 555.5, 700.01, 825.0, 829.9, 830.0, 900.0):
        for name in ('y', 'd65'):
            f = np.array(down['Y' if name == 'y' else 'D65'], np.float32)
            n = 94
            interval = np.float32(471.0) / np.float32(n)
            t = (np.float32(min(max(lam, 360.0), 830.0)) - np.float32(360.0)) / interval
            count = int(np.float32(470.0) / interval) + 1
            i = int(min(float(t), float(count - 2)))
            fr = float(t) - np.floor(float(t))
            ev.append({'table': name, 'lambda': lam, 'value': float(f[i] + np.float32(fr) * (f[i + 1] - f[i]))})
    json.dump(ev, open(os.path.join(OUT, 'spd_eval.json'), 'w'))
    write_luts(ref)


def read_luts(ref):
    text = open(os.path.join(ref, 'src/base/scattering/precomputed_table.h')).read()
    out = {}
    for name in ('DielectricLobe', 'DielectricInvLobe', 'SpecularLobe', 'PureReflectionLobe'):
        m = re.search(r'const\s+(float2|float)\s+%s_Table\[(\d+)\]\s*=\s*\{(.*?)\};' % name, text, re.S)
        body = m.group(3)
        if m.group(1) == 'float2':
            pairs = re.findall(r'float2\(\s*([-+0-9.eE]+)f?\s*,\s*([-+0-9.eE]+)f?\s*\)', body)
            vals = np.array([[float(a), float(b)] for a, b in pairs], np.float32)
        else:
            vals = np.array([float(x.rstrip('f')) for x in re.findall(r'[-+]?\d*\.\d+(?:[eE][-+]?\d+)?f?', body)],
                            np.float32)
        assert vals.shape[0] == int(m.group(2)), (name, vals.shape)
        out[name] = vals
    return out


def write_luts(ref):
    t = read_luts(ref)
    sub = [0, 5, 10, 15, 20, 25, 31]
    res = {'subgrid': sub, 'PureReflectionLobe': t['PureReflectionLobe'].tolist()}
    for name in ('DielectricLobe', 'DielectricInvLobe', 'SpecularLobe'):
        cells = []
        for z in sub:
            for y in sub:
                for x in sub:
                    v = t[name][(z * 32 + y) * 32 + x]
                    cells.append([x, y, z] + np.atleast_1d(v).astype(float).tolist())
        res[name] = cells
    json.dump(res, open(os.path.join(OUT, 'albedo_luts.json'), 'w'))


if __name__ == '__main__':
    main()
