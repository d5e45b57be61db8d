"""ORACLE — test infrastructure only.

The oracle's own scene ingestion: a vision_scene.json document -> the flat
arrays that the oracle's C++ restatement (oracle.cpp, `oracle_scene`) reads,
computed here from the reference's definitions without loading the rendering
library.  The record layouts are the flat scene format of
include/vision_b200.h (VS_EXPORT_*), the format both sides agree on; the
values are derived independently, so a scene-layer mistake in the library
(tessellation, material encoding, emitter normalisation, alias tables, the
environment warper, the sensor) shows up as a difference between
`build(doc)` and the library's export (tests/test_oracle_scene.py) instead of
being shared by both sides of every parity test.

Imported by tests/ and by bench.py's reference arm only.

Covered: shapes quad (quad.cpp:21-50), cube (cube.cpp:20-71), sphere
(sphere.cpp:17-87), inline `mesh`, the procedural `icosphere` and `grid`;
materials diffuse, black_body, metal, glass, principled_bsdf, mirror,
substrate, plastic; area emission (RGB illumination slot or the blackbody
emitter), point and spot lights; the spherical environment with the
procedural `sky` node; uniform and power light samplers; pinhole and
thin-lens sensors with box or triangle filters (the fitted filters' tables
are built by oracle.cpp itself); the independent and PCG samplers; the `pt`
integrator.  The RGB -> sigmoid-coefficient table is read from its cache
file (the reference's own table, srgb2spec.h, is a missing blob); the table's
accuracy is checked on its own by tests/test_uplift.py.
"""
import json
import math
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TABLES_INC = os.path.join(ROOT, 'vision_b200', 'csrc', 'data', 'spectral_tables.inc')
RGB2SPEC_CACHE = os.path.join(ROOT, 'vision_b200', 'data', 'srgb2spec_64.bin')

F = np.float32
INVALID = 0xffffffff
PI = F(3.14159265358979323846)

MATERIAL = np.dtype([('type', '<u4'), ('flags', '<u4'), ('spd0', '<u4'), ('spd1', '<u4'), ('coef', '<f4', 4),
                     ('p', '<f4', 8)])
LIGHT = np.dtype([('inst', '<u4'), ('first_prim', '<u4'), ('prim_count', '<u4'), ('alias_offset', '<u4'),
                  ('two_sided', '<u4'), ('kind', '<u4'), ('scale', '<f4'), ('lum_power', '<f4'), ('coef', '<f4', 4),
                  ('rgb_avg', '<f4', 4), ('shape', '<u4'), ('cos_angle', '<f4'), ('cos_start', '<f4'),
                  ('pad', '<u4'), ('pos', '<f4', 4), ('dir', '<f4', 4)])
INSTANCE = np.dtype([('mat_id', '<u4'), ('light_id', '<u4'), ('first_prim', '<u4'), ('prim_count', '<u4')])
ALIAS = np.dtype([('prob', '<f4'), ('alias', '<u4')])
CAMERA = np.dtype([('c2w', '<f4', 16), ('tan_half_fov', '<f4'), ('screen_lo_x', '<f4'), ('screen_hi_y', '<f4'),
                   ('screen_span_x', '<f4'), ('screen_span_y', '<f4'), ('filter_rx', '<f4'), ('filter_ry', '<f4'),
                   ('width', '<u4'), ('height', '<u4'), ('exposure', '<f4'), ('filter', '<u4'), ('thin_lens', '<u4'),
                   ('lens_radius', '<f4'), ('focal_distance', '<f4'), ('filter_p0', '<f4'), ('filter_p1', '<f4')])
INTEGRATOR = np.dtype([('max_depth', '<u4'), ('min_depth', '<u4'), ('rr_threshold', '<f4'), ('mis_mode', '<u4'),
                       ('spectrum_dim', '<u4'), ('scatter_pdf_dim', '<u4'), ('sampler', '<u4'), ('seed', '<u4'),
                       ('light_sampler', '<u4'), ('light_count', '<u4'), ('srgb', '<u4'), ('pad1', '<u4')])
ENV = np.dtype([('w2o', '<f4', 16), ('o2w', '<f4', 16), ('width', '<u4'), ('height', '<u4'), ('scale', '<f4'),
                ('integral', '<f4'), ('world_diameter', '<f4'), ('lum_power', '<f4'), ('pad0', '<u4'),
                ('pad1', '<u4')])
assert MATERIAL.itemsize == 64 and LIGHT.itemsize == 112 and CAMERA.itemsize == 128
assert INTEGRATOR.itemsize == 48 and ENV.itemsize == 160

# Material types and flags of the flat format.
DIFFUSE, BLACK_BODY, METAL, GLASS, PRINCIPLED, SUBSTRATE, MIX = range(7)
FLAG_DISPERSIVE, FLAG_REMAP, FLAG_CONST_FRESNEL, FLAG_PLASTIC, FLAG_ADD, FLAG_TEXTURE, FLAG_F82 = 1, 2, 4, 8, 16, 32, 64
EMIT_RGB, EMIT_BLACKBODY = 0, 1
LIGHT_AREA, LIGHT_POINT, LIGHT_SPOT, LIGHT_PROJECTOR = 0, 1, 2, 3
FILTERS = {'box': 0, 'triangle': 1, 'gaussian': 2, 'mitchell': 3, 'sinc': 4}
TONE_MAPPERS = ('linear', 'aces', 'reinhard')


class Unsupported(ValueError):
    """A scene feature the oracle's ingestion does not restate."""


# ----- data tables --------------------------------------------------------------
_TABLES = None


def tables():
    """CIE X/Y/Z/D65 at 1 nm (360..830) and the conductor eta/k curves (95
    samples), parsed from the data file generated from the reference's cie.h
    and metal_ior.inl.h."""
    global _TABLES
    if _TABLES is None:
        text = open(TABLES_INC).read()
        _TABLES = {}
        for name, body in re.findall(r'static const float (\w+)\[\d+\] = \{(.*?)\};', text, re.S):
            _TABLES[name] = np.array([float(x.rstrip('f')) for x in body.replace('\n', ' ').split(',') if x.strip()],
                                     np.float32)
    return _TABLES


def cie5():
    """SPD::create_cie_* (spd.cpp:31-38,96-110): every 5th 1-nm sample (94
    entries) and cie_y_integral (spd.cpp:14-23): trapezoids of 5 nm in FP32."""
    t = tables()
    y = t['VS_CIE_Y']
    s = F(0.0)
    for i in range(94):
        s = F(s + F(F(0.5) * F(y[5 * i] + y[5 * (i + 1)])))
    return {k: t['VS_CIE_' + k.upper()][::5][:94].copy() for k in ('x', 'y', 'z', 'd65')}, F(s * F(5.0))


_RGB2SPEC = None


def rgb2spec_table(path=RGB2SPEC_CACHE):
    """The 3 x 64^3 x 4 sigmoid-coefficient table (layout of hero.cpp's
    coefficients()[maxc][z][y][x][c])."""
    global _RGB2SPEC
    if _RGB2SPEC is None:
        if not os.path.exists(path):
            raise FileNotFoundError('RGB->spectrum table cache %s is missing (it is written the first time a scene '
                                    'with colours is loaded by the library)' % path)
        n = 3 * 64 * 64 * 64 * 4
        t = np.fromfile(path, np.float32, count=n)
        if t.size != n:
            raise ValueError('RGB->spectrum table cache %s is truncated' % path)
        _RGB2SPEC = t.reshape(3, 64, 64, 64, 4)
    return _RGB2SPEC


def luminance(rgb):
    """cie::linear_srgb_to_y (cie.h)."""
    r, g, b = (F(x) for x in rgb)
    return F(F(F(F(0.212671) * r) + F(F(0.715160) * g)) + F(F(0.072169) * b))


def decode_albedo(rgb_in):
    """RGBToSpectrumTable::decode_albedo, host path (hero.cpp:92-133)."""
    rgb = [F(min(max(F(v), F(0.0)), F(1.0))) for v in rgb_in]
    y = luminance(rgb)
    if rgb[0] == rgb[1] == rgb[2]:
        # Grey: a constant sigmoid; 0 and 1 give -inf / +inf as in the reference.
        with np.errstate(divide='ignore'):
            s = F(F(rgb[0] - F(0.5)) / F(math.sqrt(F(rgb[0] * F(F(1.0) - rgb[0])))))
        return np.array([0.0, 0.0, s, y], np.float32)
    maxc = (0 if rgb[0] > rgb[2] else 2) if rgb[0] > rgb[1] else (1 if rgb[1] > rgb[2] else 2)
    z = rgb[maxc]
    res1 = F(63.0)
    x = F(F(rgb[(maxc + 1) % 3] * res1) / z)
    yy = F(F(rgb[(maxc + 2) % 3] * res1) / z)

    def inv_ss(v):  # _inverse_smooth_step
        return F(F(0.5) - F(math.sin(F(F(math.asin(F(F(1.0) - F(F(2.0) * v)))) * F(1.0 / 3.0)))))
    zz = F(inv_ss(inv_ss(z)) * res1)
    xi, yi, zi = (min(int(v), 62) for v in (x, yy, zz))
    dx, dy, dz = F(x - F(xi)), F(yy - F(yi)), F(zz - F(zi))
    tab = rgb2spec_table()

    def lerp(t, a, b):
        return F(a + F(t * F(b - a)))
    out = np.zeros(4, np.float32)
    for i in range(3):
        def co(ox, oy, oz):
            return tab[maxc, zi + oz, yi + oy, xi + ox, i]
        out[i] = lerp(dz, lerp(dy, lerp(dx, co(0, 0, 0), co(1, 0, 0)), lerp(dx, co(0, 1, 0), co(1, 1, 0))),
                      lerp(dy, lerp(dx, co(0, 0, 1), co(1, 0, 1)), lerp(dx, co(0, 1, 1), co(1, 1, 1))))
    out[3] = y
    return out


def decode_unbound(rgb_in):
    """RGBToSpectrumTable::decode_unbound (hero.cpp:135-141)."""
    rgb = [max(F(v), F(0.0)) for v in rgb_in]
    scale = F(F(2.0) * max(rgb))
    q = [F(0.0) if scale == 0 else F(v / scale) for v in rgb]
    c = decode_albedo(q)
    c[3] = scale
    return c


# ----- alias tables ------------------------------------------------------------------
def alias_build(weights):
    """AliasTable::build (warpers/alias.h:86-122): Vose's method with an FP64
    sum, FP32 probabilities and the over/under stacks popped from the back;
    PMF = f / (integral * n) (alias.h:51-53).  Returns (table, pmf, integral)."""
    w = np.asarray(weights, np.float32)
    n = w.size
    total = float(np.sum(w.astype(np.float64)))
    ratio = n / total
    prob = (w.astype(np.float64) * ratio).astype(np.float32)
    alias = np.arange(n, dtype=np.uint32)
    over = [i for i in range(n) if prob[i] > 1.0]
    under = [i for i in range(n) if not prob[i] > 1.0]
    p = [F(x) for x in prob]
    while over and under:
        o = over.pop()
        u = under.pop()
        p[o] = F(p[o] - F(F(1.0) - p[u]))
        alias[u] = o
        if p[o] > 1.0:
            over.append(o)
        elif p[o] < 1.0:
            under.append(o)
    for i in over + under:
        p[i] = F(1.0)
        alias[i] = i
    table = np.zeros(n, ALIAS)
    table['prob'] = p
    table['alias'] = alias
    integral = F(total / n)
    pmf = (w / F(integral * F(n))) if integral > 0 else np.zeros(n, np.float32)
    return table, pmf.astype(np.float32), integral


def alias_distribution(table):
    """Probability of each entry that an alias table draws (its PMF), for
    comparing two tables built with different stack orders."""
    n = table.size
    d = np.asarray(table['prob'], np.float64) / n
    np.add.at(d, np.asarray(table['alias'], np.int64), (1.0 - np.asarray(table['prob'], np.float64)) / n)
    return d


# ----- transforms ----------------------------------------------------------------------
def _mat_mul(a, b):
    # Column-by-column FP32 product with the terms summed in order k = 0..3.
    r = np.zeros((4, 4), np.float32)
    for c in range(4):
        for row in range(4):
            s = F(0.0)
            for k in range(4):
                s = F(s + F(a[row, k] * b[k, c]))
            r[row, c] = s
    return r


def _translate(t):
    m = np.eye(4, dtype=np.float32)
    m[:3, 3] = t
    return m


def _scale(s):
    return np.diag(np.array([s[0], s[1], s[2], 1.0], np.float32))


def _rot(axis, deg):
    """Right-handed rotation by `deg` degrees about the unit x, y or z axis or
    an arbitrary axis (Rodrigues), FP32."""
    a = F(F(deg) * PI / F(180.0))
    c, s = F(math.cos(a)), F(math.sin(a))
    k = np.asarray(axis, np.float32)
    k = (k * F(F(1.0) / F(math.sqrt(F(F(F(k[0] * k[0]) + F(k[1] * k[1])) + F(k[2] * k[2])))))).astype(np.float32)
    m = np.eye(4, dtype=np.float32)
    for j in range(3):
        e = np.zeros(3, np.float32)
        e[j] = 1.0
        kxe = np.array([k[1] * e[2] - k[2] * e[1], k[2] * e[0] - k[0] * e[2], k[0] * e[1] - k[1] * e[0]], np.float32)
        col = (e * c + kxe * s + k * F(F(F(1.0) - c) * k[j])).astype(np.float32)
        m[:3, j] = col
    return m


def _look_at(pos, target, up):
    pos, target, up = (np.asarray(v, np.float32) for v in (pos, target, up))
    f = _normalize(target - pos)
    r = _normalize(_cross(f, up))
    u = _cross(r, f)
    m = np.eye(4, dtype=np.float32)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = r, u, f, pos
    return m


def _cross(a, b):
    return np.array([F(a[1] * b[2]) - F(a[2] * b[1]), F(a[2] * b[0]) - F(a[0] * b[2]),
                     F(a[0] * b[1]) - F(a[1] * b[0])], np.float32)


def _normalize(v):
    v = np.asarray(v, np.float32)
    d = F(F(F(v[0] * v[0]) + F(v[1] * v[1])) + F(v[2] * v[2]))
    return (v * F(F(1.0) / F(math.sqrt(d)))).astype(np.float32)


def _f3(j, default):
    if isinstance(j, (list, tuple)) and len(j) >= 3:
        return np.array(j[:3], np.float32)
    return np.array(default, np.float32)


def transform(t):
    """TransformDesc::init (node_desc.cpp:26-52): matrix4x4 (columns), look_at,
    Euler, trs; returns a row-major FP32 4x4."""
    if not t:
        return np.eye(4, dtype=np.float32)
    typ = t.get('type', 'matrix4x4')
    p = t.get('param', {})
    if typ == 'matrix4x4':
        if 'matrix4x4' not in p:
            return np.eye(4, dtype=np.float32)
        return np.array(p['matrix4x4'], np.float32).T.copy()
    if typ == 'look_at':
        return _look_at(_f3(p.get('position'), (0, 0, 0)), _f3(p.get('target_pos'), (0, 0, 1)),
                        _f3(p.get('up'), (0, 1, 0)))
    if typ == 'Euler':
        m = _mat_mul(_translate(_f3(p.get('position'), (0, 0, 0))), _rot((1, 0, 0), p.get('pitch', 0.0)))
        m = _mat_mul(m, _rot((0, 0, 1), p.get('roll', 0.0)))
        return _mat_mul(m, _rot((0, 1, 0), p.get('yaw', 0.0)))
    if typ == 'trs':
        r = p.get('r', [1.0, 0.0, 0.0, 0.0])
        m = _mat_mul(_translate(_f3(p.get('t'), (0, 0, 0))), _rot(r[:3], r[3]))
        return _mat_mul(m, _scale(_f3(p.get('s'), (1, 1, 1))))
    raise Unsupported('transform type ' + typ)


def xform_points(m, p):
    """Affine point transform in FP32, terms summed in column order."""
    p = np.asarray(p, np.float32)
    out = np.empty_like(p)
    for r in range(3):
        out[:, r] = ((m[r, 0] * p[:, 0] + m[r, 1] * p[:, 1]) + m[r, 2] * p[:, 2]) + m[r, 3]
    w = ((m[3, 0] * p[:, 0] + m[3, 1] * p[:, 1]) + m[3, 2] * p[:, 2]) + m[3, 3]
    scale = w != 1.0
    if scale.any():
        out[scale] = out[scale] / w[scale, None]
    return out


def xform_normals(m, n):
    """Normals through the inverse transpose of the upper 3x3 (FP64, rounded
    once); zero normals stay zero."""
    n = np.asarray(n, np.float32)
    inv_t = np.linalg.inv(m[:3, :3].astype(np.float64)).T
    out = (n.astype(np.float64) @ inv_t.T).astype(np.float32)
    zero = ~n.any(1)
    out[zero] = 0.0
    return out


# ----- shapes --------------------------------------------------------------------------
def quad(p):
    """Quad::init (quad.cpp:21-50): four corners in the xz plane, every normal
    the unnormalised cross((p0 - p2), (p1 - p2)), triangles (0,1,2), (2,1,3)."""
    w, h = F(F(p.get('width', 1.0)) / F(2)), F(F(p.get('height', 1.0)) / F(2))
    P = np.array([[w, 0, h], [w, 0, -h], [-w, 0, h], [-w, 0, -h]], np.float32)
    ng = _cross(P[0] - P[2], P[1] - P[2])
    N = np.tile(ng, (4, 1))
    UV = np.array([[1, 1], [1, 0], [0, 1], [0, 0]], np.float32)
    return P, N, UV, np.array([0, 1, 2, 2, 1, 3], np.uint32)


def cube(p):
    """Cube::init (cube.cpp:20-71): 24 vertices, four per face, 12 triangles."""
    x, y, z = F(p.get('x', 1.0)), F(p.get('y', 1.0)), F(p.get('z', 1.0))
    y = x if y == 0 else y
    z = y if z == 0 else z
    x, y, z = F(x / F(2)), F(y / F(2)), F(z / F(2))
    faces = [  # corners and the face normal, in the reference's order
        ([(-x, -y, z), (x, -y, z), (-x, y, z), (x, y, z)], (0, 0, 1)),
        ([(-x, y, -z), (x, y, -z), (-x, -y, -z), (x, -y, -z)], (0, 0, -1)),
        ([(-x, y, z), (x, y, z), (-x, y, -z), (x, y, -z)], (0, 1, 0)),
        ([(-x, -y, z), (x, -y, z), (-x, -y, -z), (x, -y, -z)], (0, -1, 0)),
        ([(x, -y, z), (x, y, z), (x, y, -z), (x, -y, -z)], (1, 0, 0)),
        ([(-x, -y, z), (-x, y, z), (-x, y, -z), (-x, -y, -z)], (-1, 0, 0))]
    P = np.array([c for cs, _ in faces for c in cs], np.float32)
    N = np.array([n for _, n in faces for _ in range(4)], np.float32)
    UV = np.array([(0, 0), (1, 0), (0, 1), (1, 1), (0, 1), (1, 1), (0, 0), (1, 0), (0, 1), (1, 1), (0, 0), (1, 0),
                   (0, 1), (1, 1), (0, 0), (1, 0), (0, 1), (1, 1), (1, 0), (0, 0), (0, 1), (1, 1), (1, 0), (0, 0)],
                  np.float32)
    tri = [(0, 1, 3), (0, 3, 2), (6, 5, 7), (4, 5, 6), (10, 9, 11), (8, 9, 10), (13, 14, 15), (13, 12, 14),
           (18, 17, 19), (17, 16, 19), (21, 22, 23), (20, 21, 23)]
    return P, N, UV, np.array(tri, np.uint32).ravel()


def sphere(p):
    """Sphere (sphere.cpp:17-87): pole at +y, sub_div - 1 rings of 2 sub_div
    vertices from the top, pole at -y; top fan, bands, bottom fan."""
    radius, n = F(p.get('radius', 1.0)), int(p.get('sub_div', 60))
    if n < 2:
        raise Unsupported('sphere sub_div < 2')
    m = 2 * n
    P, N, UV = [(0, radius, 0)], [(0, 1, 0)], [(0, 0)]
    for i in range(1, n):
        v = F(F(i) / F(n))
        theta = F(PI * v)
        y, r = F(radius * F(math.cos(theta))), F(radius * F(math.sin(theta)))
        for j in range(m):
            u = F(F(j) / F(m))
            phi = F(F(u * F(2.0)) * PI)
            q = (r, y, F(0)) if j == 0 else (F(F(math.cos(phi)) * r), y, F(F(math.sin(phi)) * r))
            P.append(q)
            N.append(tuple(_normalize(np.array(q, np.float32))))
            UV.append((F(0) if j == 0 else u, v))
    P.append((0, -radius, 0))
    N.append((0, -1, 0))
    UV.append((0, 1))
    idx = []
    for i in range(m):
        idx += [0, (i + 1) % m + 1, i + 1]
    for i in range(n - 2):
        vs = 1 + i * m
        for j in range(m):
            if j != m - 1:
                idx += [vs, vs + 1, vs + m, vs + 1, vs + m + 1, vs + m]
            else:
                idx += [vs, vs + 1 - m, vs + m, vs + 1 - m, vs + 1, vs + m]
            vs += 1
    last = len(P) - 1
    for i in range(m):
        idx += [last, last - ((1 + i) % m + 1), last - (i + 1)]
    return (np.array(P, np.float32), np.array(N, np.float32), np.array(UV, np.float32), np.array(idx, np.uint32))


def inline_mesh(p):
    P = np.array(p['positions'], np.float32).reshape(-1, 3)
    N = np.array(p['normals'], np.float32).reshape(-1, 3) if p.get('normals') else np.zeros_like(P)
    UV = np.array(p['uvs'], np.float32).reshape(-1, 2) if p.get('uvs') else np.zeros((len(P), 2), np.float32)
    return P, N, UV, np.array(p['indices'], np.uint32)


def _noise_hash(x, y, z, seed):
    h = (x.astype(np.uint32) * np.uint32(0x8da6b343)) ^ (y.astype(np.uint32) * np.uint32(0xd8163841)) ^ \
        (z.astype(np.uint32) * np.uint32(0xcb1ab31f)) ^ np.uint32((seed * 0x165667b1) & 0xffffffff)
    h = h ^ (h >> np.uint32(13))
    h = h * np.uint32(0x5bd1e995)
    h = h ^ (h >> np.uint32(15))
    return (h & np.uint32(0xffffff)).astype(np.float32) * F(2.0 / 16777215.0) - F(1.0)


def value_noise(p, seed):
    """Lattice value noise in [-1, 1]: hashed lattice values, trilinear
    interpolation with smoothstep weights (the `displacement` of the
    procedural icosphere)."""
    fl = np.floor(p)
    i = fl.astype(np.int64).astype(np.int32)
    t = (p - fl).astype(np.float32)
    t = (t * t * (F(3.0) - F(2.0) * t)).astype(np.float32)
    with np.errstate(over='ignore'):
        def h(dx, dy, dz):
            return _noise_hash(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)

        def l(tt, a, b):
            return a + tt * (b - a)
        c00 = l(t[:, 0], h(0, 0, 0), h(1, 0, 0))
        c10 = l(t[:, 0], h(0, 1, 0), h(1, 1, 0))
        c01 = l(t[:, 0], h(0, 0, 1), h(1, 0, 1))
        c11 = l(t[:, 0], h(0, 1, 1), h(1, 1, 1))
        return l(t[:, 2], l(t[:, 1], c00, c10), l(t[:, 1], c01, c11)).astype(np.float32)


def _normalize_rows(v):
    d = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    return (v * (F(1.0) / np.sqrt(d))[:, None]).astype(np.float32)


def icosphere(p):
    """Procedural displaced icosphere: an icosahedron subdivided `subdivisions`
    times (each edge midpoint projected to the unit sphere, triangles split
    into four), radius times (1 + amplitude * value_noise(frequency * v)),
    vertex normals the sums of the faces' cross((p0 - p2), (p1 - p2)),
    spherical uv."""
    sub = int(p.get('subdivisions', 4))
    if sub > 9:
        raise Unsupported('icosphere subdivisions > 9')
    radius = F(p.get('radius', 1.0))
    d = p.get('displacement', {}) or {}
    amp, freq, seed = F(d.get('amplitude', 0.0)), F(d.get('frequency', 4.0)), int(d.get('seed', 1))
    t = F(F(F(1.0) + F(math.sqrt(F(5.0)))) / F(2.0))
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float32)
    v = _normalize_rows(v)
    f = np.array([0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                  3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1],
                 np.int64).reshape(-1, 3)
    verts = [v]
    nv = len(v)
    for _ in range(sub):
        # Midpoints are numbered in the order the triangles first meet them:
        # edges (a, b), (b, c), (c, a) of each triangle in turn.
        e = np.stack([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 1).reshape(-1, 2)
        key = np.minimum(e[:, 0], e[:, 1]) * (1 << 32) + np.maximum(e[:, 0], e[:, 1])
        uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
        order = np.argsort(first, kind='stable')
        rank = np.empty_like(order)
        rank[order] = np.arange(order.size)
        mid_id = nv + rank[inv]
        all_v = np.concatenate(verts)
        a, b = e[first[order], 0], e[first[order], 1]
        mids = _normalize_rows(((all_v[a] + all_v[b]) * F(0.5)).astype(np.float32))
        verts.append(mids)
        nv += len(mids)
        m = mid_id.reshape(-1, 3)
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.stack([f[:, 0], ab, ca, f[:, 1], bc, ab, f[:, 2], ca, bc, ab, bc, ca], 1).reshape(-1, 3)
    v = np.concatenate(verts)
    r = (radius * (F(1.0) + amp * value_noise((v * freq).astype(np.float32), seed))).astype(np.float32)
    P = (v * r[:, None]).astype(np.float32)
    theta = np.arccos(np.clip(v[:, 1].astype(np.float64), -1.0, 1.0)).astype(np.float32)
    phi = np.arctan2(v[:, 2].astype(np.float64), v[:, 0].astype(np.float64)).astype(np.float32)
    UV = np.stack([phi * F(0.15915494309189533577) + F(0.5), theta * F(0.31830988618379067154)], 1)
    N = np.zeros_like(P)
    p0, p1, p2 = P[f[:, 0]], P[f[:, 1]], P[f[:, 2]]
    a, b = p0 - p2, p1 - p2
    fn = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                   a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)
    for k in range(3):
        np.add.at(N, f[:, k], fn)
    return P, N, UV.astype(np.float32), f.astype(np.uint32).ravel()


def grid(p):
    """Procedural ground grid in the xz plane facing +y: nx x nz quads, two
    triangles (c, b, a), (c, d, b) each."""
    nx, nz = int(p.get('nx', 1)), int(p.get('nz', 1))
    sx, sz = F(p.get('size_x', 1.0)), F(p.get('size_z', 1.0))
    j, i = np.mgrid[0:nz + 1, 0:nx + 1]
    u = (i.astype(np.float32) / F(nx)).ravel()
    w = (j.astype(np.float32) / F(nz)).ravel()
    P = np.stack([(u - F(0.5)) * sx, np.zeros_like(u), (w - F(0.5)) * sz], 1).astype(np.float32)
    N = np.tile(np.array([0, 1, 0], np.float32), (len(P), 1))
    UV = np.stack([u, w], 1)
    jj, ii = np.mgrid[0:nz, 0:nx]
    a = (jj * (nx + 1) + ii).ravel()
    b, c = a + 1, a + nx + 1
    d = c + 1
    idx = np.stack([c, b, a, c, d, b], 1).astype(np.uint32).ravel()
    return P, N, UV, idx


SHAPES = {'quad': quad, 'cube': cube, 'sphere': sphere, 'mesh': inline_mesh, 'icosphere': icosphere, 'grid': grid}


# ----- spectra of slots ---------------------------------------------------------------------
def _node_type(n):
    """ShaderNodeDesc::init (node_desc.cpp:292-320): {"type", "param"}, or
    the parameters inline, where an object naming a file is an image node."""
    if not isinstance(n, dict):
        return None
    if 'param' in n:
        return n.get('type', 'number')
    return n.get('type', 'image' if 'fn' in n else 'number')


def _node_param(n):
    return n.get('param', {}) or {} if 'param' in n else n


def _slot(j):
    """SlotDesc::init (node_desc.cpp:127-150): a number, a list, a
    {"channels", "node"} pair or a number/constant node, as a float list."""
    if isinstance(j, (int, float)):
        return [float(j)]
    if isinstance(j, list):
        return [float(x) for x in j]
    if isinstance(j, dict):
        if 'channels' in j:
            return _slot(j['node'])
        t = _node_type(j)
        if t in ('number', 'constant'):
            return _slot(j.get('param', j).get('value'))
        raise Unsupported('shader node ' + t)
    return []


def _slot_rgb(j, default):
    v = _slot(j) if j is not None else []
    if not v:
        return [F(default)] * 3
    if len(v) == 1:
        return [F(v[0])] * 3
    return [F(v[0]), F(v[1]), F(v[2] if len(v) > 2 else v[1])]


def _slot_scalar(j, default):
    v = _slot(j) if j is not None else []
    return F(v[0] if v else default)


def _node(j):
    return j['node'] if isinstance(j, dict) and 'channels' in j else j


def srgb_to_linear(c):
    """The sRGB transfer function removed (IEC 61966-2-1), in float32."""
    c = np.asarray(c, np.float32)
    hi = np.power(((c + F(0.055)) / F(1.055)).astype(np.float32), F(2.4)).astype(np.float32)
    return np.where(c <= F(0.04045), (c / F(12.92)).astype(np.float32), hi).astype(np.float32)


def load_texels(node, base_dir):
    """The file of an `image` node (ImagePool::load_texture,
    image_pool.cpp:13-35) as (H, W, 4) float32 linear RGB texels and 0: the
    path relative to the scene's folder, the colour space "srgb" by default
    ("linear" for Radiance HDR) with its transfer function removed, grey
    replicated to RGB, alpha dropped.  Decoded by OpenCV: PNG and Radiance
    HDR exactly as the library does; baseline JPEG to within a few levels of
    8 bits (libjpeg's integer IDCT against the library's float IDCT)."""
    os.environ.setdefault('OPENCV_IO_ENABLE_OPENEXR', '1')
    import cv2
    p = _node_param(node)
    fn = p.get('fn', '')
    if not fn:
        raise ValueError('image node without fn')
    path = fn if os.path.isabs(fn) or not base_dir else os.path.join(base_dir, fn)
    ext = fn.rsplit('.', 1)[-1].lower() if '.' in fn else ''
    if ext not in ('png', 'jpg', 'jpeg', 'hdr', 'exr'):
        raise Unsupported('image file format ' + ext)
    cs = p.get('color_space') or ('linear' if ext in ('hdr', 'exr') else 'srgb')
    if cs not in ('srgb', 'linear'):
        raise Unsupported('image colour space ' + cs)
    im = cv2.imread(path, cv2.IMREAD_UNCHANGED)
    if im is None:
        raise ValueError('cannot decode ' + path)
    if im.dtype == np.uint8:
        f = im.astype(np.float32) / F(255.0)
    elif im.dtype == np.uint16:
        f = im.astype(np.float32) / F(65535.0)
    else:
        f = im.astype(np.float32)
    if f.ndim == 2:
        rgb = np.repeat(f[..., None], 3, axis=2)
    elif f.shape[2] == 2:
        rgb = np.repeat(f[..., :1], 3, axis=2)
    else:
        rgb = f[..., 2::-1] if f.shape[2] >= 3 else f
    rgb = srgb_to_linear(rgb) if cs == 'srgb' else rgb
    tex = np.zeros(rgb.shape[:2] + (4,), np.float32)
    tex[..., :3] = rgb
    return tex


def _to_list(f):
    """SPD::to_list (spd.h:41-47): every 5 nm from 360 nm below 830 nm."""
    out, l = [], F(360.0)
    while l < F(830.0):
        out.append(f(l))
        l = F(l + F(5.0))
    return np.array(out, np.float32)


def sellmeier(name):
    """Glass IOR curves of glass.cpp:104-134 (BK7, LASF9 Sellmeier fits)."""
    if name == 'LASF9':
        c = (2.00029547, 0.298926886, 1.80691843, 0.0121426017, 0.0538736236, 156.530829)
    else:
        c = (1.03961212, 0.231792344, 1.01046945, 0.00600069867, 0.0200179144, 103.560653)
    b1, b2, b3, c1, c2, c3 = (F(x) for x in c)

    def n(lam):
        l = F(lam / F(1000.0))
        l2 = F(l * l)
        f = F(F(F(b1 * l2) / F(l2 - c1)) + F(F(b2 * l2) / F(l2 - c2))) + F(F(b3 * l2) / F(l2 - c3))
        return F(math.sqrt(F(f + F(1.0))))
    return _to_list(n)


def cauchy(A, B):
    """Cauchy dispersion n = A + B / lambda^2 (lambda in micrometres) as an
    ior spd slot (the reference has no Cauchy curve)."""
    A, B = F(A), F(B)
    return _to_list(lambda lam: F(A + F(B / F(F(lam / F(1000.0)) * F(lam / F(1000.0))))))


def planck(lam_nm, T):
    """Planck's law, W / (m^2 sr m), lambda in nm (optics.h:82-90)."""
    c, h, kb = 299792458.0, 6.62606957e-34, 1.3806488e-23
    l = lam_nm * 1e-9
    return (2.0 * h * c * c) / (l ** 5 * (math.exp((h * c) / (l * kb * T)) - 1.0))


def blackbody_average(T):
    """Linear sRGB of the blackbody emitter's spectrum normalised to a peak
    of one (the Planck curve at Wien's peak), and 1 / that peak."""
    t = tables()
    inv_peak = F(1.0 / planck(2.8977721e-3 / T * 1e9, T))
    lam = 360.0 + np.arange(471)
    e = np.array([planck(l, T) for l in lam]) * float(inv_peak)
    _, yi = cie5()
    xyz = [float(np.sum(e * t[k].astype(np.float64))) / float(yi) for k in ('VS_CIE_X', 'VS_CIE_Y', 'VS_CIE_Z')]
    X, Y, Z = xyz
    rgb = [3.240479 * X - 1.537150 * Y - 0.498535 * Z, -0.969256 * X + 1.875991 * Y + 0.041556 * Z,
           0.055648 * X - 0.204043 * Y + 1.057311 * Z]
    return np.array(rgb, np.float32), inv_peak


# ----- the scene ----------------------------------------------------------------------------
class _Builder:
    def __init__(self, doc, base_dir):
        self.doc = doc
        self.base_dir = base_dir
        self.pos, self.nrm, self.uv, self.idx, self.prim_inst = [], [], [], [], []
        self.nverts = 0
        self.nprims = 0
        self.instances, self.materials, self.lights = [], [], []
        self.mat_by_name = {}
        self.prim_alias, self.prim_pmf = [], []
        self.spd = []
        self.spd_len = 0
        self.needs_luts = False
        self.tex_texels, self.textures, self.tex_by_key, self.tex_avg = [], [], {}, []
        self.tex_len = 0

    def texture(self, node):
        """The id of an image node's texture, each file and colour space loaded once."""
        p = _node_param(node)
        key = (p.get('fn', ''), p.get('color_space', ''))
        if key not in self.tex_by_key:
            tex = load_texels(node, self.base_dir)
            H, W = tex.shape[:2]
            self.tex_by_key[key] = len(self.textures)
            self.textures.append((self.tex_len, W, H, 0))
            self.tex_texels.append(tex.reshape(-1))
            self.tex_len += W * H
            self.tex_avg.append(tex.reshape(-1, 4)[:, :3].astype(np.float64).mean(0).astype(np.float32))
        return self.tex_by_key[key]

    def colour_slot(self, j, default, r):
        """A material colour slot: a constant (sigmoid coefficients, or the
        colour itself for the RGB spectrum), an `image` node, or a `multiply`
        of an image node and a constant (math.cpp).  A texture sets flag 32,
        the id's bits in p[7] and the constant factor as RGB in coef."""
        n = _node(j)
        img, factor = None, [F(1.0)] * 3
        if _node_type(n) == 'image':
            img = n
        elif _node_type(n) == 'multiply':
            q = n.get('param', {}) or {}
            lhs, rhs = _node(q.get('lhs')), _node(q.get('rhs'))
            li = _node_type(lhs) == 'image'
            ri = _node_type(rhs) == 'image'
            if li == ri:
                raise Unsupported('multiply node other than an image times a constant')
            img = lhs if li else rhs
            factor = _slot_rgb(q.get('rhs') if li else q.get('lhs'), 1.0)
        if img is None:
            r['coef'] = self.colour(_slot_rgb(j, default))
            return
        tid = self.texture(img)
        r['flags'] |= FLAG_TEXTURE
        r['p'][7] = np.array([tid], np.uint32).view(np.float32)[0]
        r['coef'] = [factor[0], factor[1], factor[2], 0.0]

    def colour(self, rgb):
        if self.srgb:
            return np.array([rgb[0], rgb[1], rgb[2], 0.0], np.float32)
        return decode_albedo(rgb)

    def add_spd(self, v):
        off = self.spd_len
        self.spd.append(np.concatenate([[F(len(v))], np.asarray(v, np.float32)]).astype(np.float32))
        self.spd_len += len(v) + 1
        return off

    def material(self, m):
        """Material records (diffuse.cpp, black_body.cpp, metal.cpp, glass.cpp,
        principled_bsdf.cpp, mirror.cpp, substrate.cpp, plastic.cpp, mix.cpp,
        add.cpp)."""
        t, p = m.get('type', 'diffuse'), m.get('param', {}) or {}
        r = np.zeros(1, MATERIAL)[0]
        r['spd0'] = r['spd1'] = INVALID

        def alphas(a, aniso):
            if abs(aniso) <= F(1e-4):
                return a, a
            return (F(a / F(F(1) + aniso)) if aniso < 0 else F(a * F(F(1) - aniso)),
                    F(a * F(F(1) + aniso)) if aniso < 0 else F(a / F(F(1) - aniso)))

        def clamp(x, lo, hi):
            return F(min(max(F(x), F(lo)), F(hi)))
        if t in ('mix', 'add'):
            # MixMaterial / AddMaterial (mix.cpp:20-68, add.cpp:12-59): the two
            # inline material nodes (node_desc.cpp:155-161) as records of their
            # own, named after this one, then this record with their indices.
            r['type'] = MIX
            if t == 'add':
                r['flags'] |= FLAG_ADD
            else:
                r['p'][0] = _slot_scalar(p.get('frac'), 0.5)
            for k in (0, 1):
                c = p.get('mat%d' % k)
                if not isinstance(c, dict):
                    raise ValueError('material %s: missing mat%d' % (m.get('name', ''), k))
                if c.get('type', 'diffuse') in ('mix', 'add', 'black_body'):
                    raise Unsupported('%s inside a mix / add material' % c.get('type'))
                c = dict(c, name='%s/mat%d' % (m.get('name', ''), k))
                self.material(c)
                r['spd0' if k == 0 else 'spd1'] = len(self.materials) - 1
        elif t == 'diffuse':
            r['type'] = DIFFUSE
            self.colour_slot(p.get('color'), 0.5, r)
        elif t == 'black_body':
            r['type'] = BLACK_BODY
        elif t in ('metal', 'mirror'):
            r['type'] = METAL
            if t == 'metal':
                name = p.get('material_name', '')
                tab = tables()
                key = {'Ag': 'AG', 'Al': 'AL', 'Au': 'AU', 'Cu': 'CU', 'CuZn': 'CUZN', 'Fe': 'FE', 'Ti': 'TI',
                       'V': 'V', 'VN': 'VN', 'Li': 'LI'}.get(name, 'AG')
                r['spd0'] = self.add_spd(tab['VS_METAL_%s_ETA' % key])
                r['spd1'] = self.add_spd(tab['VS_METAL_%s_K' % key])
                rough = clamp(_slot_scalar(p.get('roughness'), 0.01), 0.0001, 1.0)
            else:
                r['flags'] |= FLAG_CONST_FRESNEL
                self.colour_slot(p.get('color'), 1.0, r)
                rough = clamp(_slot_scalar(p.get('roughness'), 0.001), 0.0001, 1.0)
            aniso = clamp(_slot_scalar(p.get('anisotropic'), 0.0), -0.9, 0.9)
            a = F(rough * rough) if p.get('remapping_roughness', True) else rough
            r['p'][0], r['p'][1] = alphas(a, aniso)
            self.needs_luts = True
        elif t == 'metallic':
            # MetallicMaterial (metallic.cpp:26-60): colour, edge tint (an
            # albedo in p[2..4]), roughness in [0.01, 1] always remapped.
            r['type'] = METAL
            r['flags'] |= FLAG_F82
            self.colour_slot(p.get('color'), 1.0, r)
            r['p'][2:5] = self.colour(_slot_rgb(p.get('edge_tint'), 1.0))[:3]
            rough = clamp(_slot_scalar(p.get('roughness'), 0.5), 0.01, 1.0)
            aniso = clamp(_slot_scalar(p.get('anisotropic'), 0.0), -0.9, 0.9)
            r['p'][0], r['p'][1] = alphas(F(rough * rough), aniso)
            self.needs_luts = True
        elif t == 'glass':
            r['type'] = GLASS
            self.colour_slot(p.get('color'), 1.0, r)
            ior = p.get('ior')
            node = _node(ior)
            curve = None
            if p.get('material_name'):
                curve = sellmeier(p['material_name'])
            elif isinstance(node, dict) and node.get('type') == 'spd':
                curve = np.array((node.get('param') or node)['value'], np.float32)
            elif isinstance(node, dict) and node.get('type') == 'cauchy':
                cp = node.get('param', {})
                curve = cauchy(cp.get('A', 1.5), cp.get('B', 0.0))
            if curve is not None:
                r['spd0'] = self.add_spd(curve)
                r['flags'] |= FLAG_DISPERSIVE
            else:
                r['p'][2] = _slot_scalar(ior, 1.5)
            rough = clamp(_slot_scalar(p.get('roughness'), 0.5), 0.01, 1.0)
            aniso = clamp(_slot_scalar(p.get('anisotropic'), 0.0), -0.9, 0.9)
            a = F(rough * rough) if p.get('remapping_roughness', True) else rough
            r['p'][0], r['p'][1] = alphas(a, aniso)
            self.needs_luts = True
        elif t == 'principled_bsdf':
            r['type'] = PRINCIPLED
            self.colour_slot(p.get('color'), 1.0, r)
            rough = clamp(_slot_scalar(p.get('roughness'), 0.5), 0.0001, 1.0)
            aniso = _slot_scalar(p.get('anisotropic'), 0.0)
            aspect = F(math.sqrt(F(F(1.0) - F(aniso * F(0.9)))))
            r['p'][0] = max(F(0.001), F(F(rough * rough) / aspect))
            r['p'][1] = max(F(0.001), F(F(rough * rough) * aspect))
            r['p'][2] = _slot_scalar(p.get('metallic'), 0.0)
            r['p'][3] = _slot_scalar(p.get('ior'), 1.5)
            r['p'][4:7] = self.colour(_slot_rgb(p.get('spec_tint'), 1.0))[:3]
            # Sheen, coat and transmission layers (initialize_slots,
            # principled_bsdf.cpp:287-302) as a 12-float block of the SPD
            # table when any of their weights is non-zero.
            sw, cw, tw = (_slot_scalar(p.get(k), 0.0) for k in ('sheen_weight', 'coat_weight',
                                                                 'transmission_weight'))
            if sw != 0.0 or cw != 0.0 or tw != 0.0:
                block = [sw, _slot_scalar(p.get('sheen_roughness'), 0.5)]
                block += list(self.colour(_slot_rgb(p.get('sheen_tint'), 1.0))[:3])
                block += [cw, _slot_scalar(p.get('coat_roughness'), 0.2), _slot_scalar(p.get('coat_ior'), 1.5)]
                block += list(self.colour(_slot_rgb(p.get('coat_tint'), 1.0))[:3])
                block += [tw]
                r['spd0'] = self.add_spd(np.array(block, np.float32))
            self.needs_luts = True
        elif t in ('substrate', 'plastic'):
            r['type'] = SUBSTRATE
            if t == 'plastic':
                r['flags'] |= FLAG_PLASTIC
                r['p'][5] = clamp(_slot_scalar(p.get('ior'), 1.3), 1.003, 5.0)
            self.colour_slot(p.get('color'), 1.0, r)
            r['p'][2:5] = self.colour(_slot_rgb(p.get('spec'), 0.05))[:3]
            rough = clamp(_slot_scalar(p.get('roughness'), 0.5), 0.0001, 1.0)
            aniso = clamp(_slot_scalar(p.get('anisotropic'), 0.0), -0.9, 0.9)
            remap = p.get('remapping_roughness', True)
            ax, ay = alphas(F(rough * rough) if remap else rough, aniso)
            if remap:
                ax, ay = F(ax * ax), F(ay * ay)
            r['p'][0], r['p'][1] = clamp(ax, 0.0001, 1.0), clamp(ay, 0.0001, 1.0)
        else:
            raise Unsupported('material ' + t)
        self.mat_by_name[m.get('name', '')] = len(self.materials)
        self.materials.append(r)

    def black_body_material(self):
        if '__black_body__' not in self.mat_by_name:
            self.material({'type': 'black_body', 'name': '__black_body__', 'param': {}})
        return self.mat_by_name['__black_body__']

    def emitter(self, p, L):
        """Light::Light (light.cpp:10-17) with NumberNode::normalize
        (number.cpp:40-48): the largest RGB channel, when >= 1, folds into the
        scale; or the blackbody emitter."""
        scale = F(p['scale']) if isinstance(p.get('scale'), (int, float)) else F(1.0)
        node = _node(p.get('color'))
        if isinstance(node, dict) and node.get('type') == 'blackbody':
            T = float(node.get('param', {}).get('temperature', 6500.0))
            avg, inv_peak = blackbody_average(F(T))
            L['kind'] = EMIT_BLACKBODY
            L['coef'] = [F(T), inv_peak, 0, 0]
        else:
            rgb = _slot_rgb(p.get('color'), 1.0)
            mx = max(rgb)
            if mx >= 1.0:
                rgb = [F(c / mx) for c in rgb]
                scale = F(scale * mx)
            L['kind'] = EMIT_RGB
            L['coef'] = decode_unbound(rgb)
            avg = np.array(rgb, np.float32)
        L['scale'] = scale
        L['rgb_avg'][:3] = (avg * scale).astype(np.float32)

    def shape(self, sh):
        t, p = sh.get('type'), sh.get('param', {}) or {}
        if t not in SHAPES:
            raise Unsupported('shape ' + str(t))
        P, N, UV, idx = SHAPES[t](p)
        m = transform(p.get('transform'))
        P = xform_points(m, P)
        N = xform_normals(m, N)
        emission = p.get('emission')
        mname = p.get('material', '')
        if mname:
            if mname not in self.mat_by_name:
                raise ValueError('unknown material ' + mname)
            mat = self.mat_by_name[mname]
        else:
            mat = self.black_body_material()
        inst = np.zeros(1, INSTANCE)[0]
        inst['mat_id'], inst['light_id'] = mat, INVALID
        inst['first_prim'], inst['prim_count'] = self.nprims, len(idx) // 3
        base = self.nverts
        self.pos.append(P)
        self.nrm.append(N)
        self.uv.append(UV)
        self.idx.append(idx.astype(np.uint32) + np.uint32(base))
        self.prim_inst.append(np.full(len(idx) // 3, len(self.instances), np.uint32))
        self.nverts += len(P)
        self.nprims += len(idx) // 3
        if emission:
            if emission.get('type', 'area') != 'area':
                raise Unsupported('emission ' + emission.get('type'))
            ep = emission.get('param', {}) or {}
            L = np.zeros(1, LIGHT)[0]
            L['inst'], L['first_prim'], L['prim_count'] = len(self.instances), inst['first_prim'], inst['prim_count']
            L['two_sided'] = 1 if ep.get('two_sided', False) else 0
            L['shape'] = LIGHT_AREA
            self.emitter(ep, L)
            # AreaLight::prepare: per-triangle areas, alias table (area.cpp:33-60).
            tri = idx.reshape(-1, 3)
            a, b = P[tri[:, 0]] - P[tri[:, 2]], P[tri[:, 1]] - P[tri[:, 2]]
            cr = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                           a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)
            area = (F(0.5) * np.sqrt((cr[:, 0] * cr[:, 0] + cr[:, 1] * cr[:, 1]) + cr[:, 2] * cr[:, 2])).astype(
                np.float32)
            tab, pmf, _ = alias_build(area)
            L['alias_offset'] = sum(len(x) for x in self.prim_alias)
            self.prim_alias.append(tab)
            self.prim_pmf.append(pmf)
            total = F(0.0)
            for x in area:
                total = F(total + x)
            # AreaLight::power (area.cpp:87-89).
            k = F(F(2.0) if L['two_sided'] else F(1.0))
            power = [F(F(k * L['rgb_avg'][c]) * F(total * PI)) if L['two_sided'] else F(L['rgb_avg'][c] *
                                                                                          F(total * PI))
                     for c in range(3)]
            L['lum_power'] = luminance(power)
            inst['light_id'] = len(self.lights)
            self.lights.append(L)
        self.instances.append(inst)

    def point_light(self, typ, p):
        """PointLight (point.cpp:20-43) and SpotLight (spot.cpp:19-70)."""
        L = np.zeros(1, LIGHT)[0]
        L['inst'] = L['first_prim'] = L['prim_count'] = L['alias_offset'] = INVALID
        L['shape'] = LIGHT_SPOT if typ == 'spot' else LIGHT_POINT
        self.emitter(p, L)
        L['pos'][:3] = _f3(p.get('position'), (0, 0, 0))
        avg = L['rgb_avg'][:3].astype(np.float32)
        if typ == 'point':
            L['lum_power'] = luminance(avg * F(F(4.0) * PI))
        else:
            L['dir'][:3] = _normalize(_f3(p.get('direction'), (0, 0, 1)))
            angle = F(F(min(max(F(p.get('angle', 45.0)), F(1.0)), F(89.0))) * PI / F(180.0))
            falloff = min(max(F(F(F(p.get('falloff', 10.0)) * PI) / F(180.0)), F(0.0)), angle)
            L['cos_angle'] = F(math.cos(angle))
            L['cos_start'] = F(math.cos(max(F(0.0), F(angle - falloff))))
            L['lum_power'] = luminance(avg * F(F(F(2.0) * PI) * F(F(1.0) - F(F(0.5) * F(F(angle * F(2.0)) +
                                                                                       falloff)))))
        self.lights.append(L)

    def projector(self, p):
        """Projector (projector.cpp:30-126): a delta-position light at the
        origin of o2w projecting its colour slot (an image, an image times a
        constant, or a constant colour) through a pinhole along +z; its
        16-float SPD-table block holds the world-to-light rows, the tangents
        of the half-angles and the texture id's bits."""
        L = np.zeros(1, LIGHT)[0]
        L['inst'] = L['first_prim'] = L['prim_count'] = INVALID
        L['shape'] = LIGHT_PROJECTOR
        n = _node(p.get('color'))
        img, factor = None, [F(1.0)] * 3
        if _node_type(n) == 'image':
            img = n
        elif _node_type(n) == 'multiply':
            q = n.get('param', {}) or {}
            lhs, rhs = _node(q.get('lhs')), _node(q.get('rhs'))
            li, ri = _node_type(lhs) == 'image', _node_type(rhs) == 'image'
            if li == ri:
                raise Unsupported('multiply node other than an image times a constant')
            img = lhs if li else rhs
            factor = _slot_rgb(q.get('rhs') if li else q.get('lhs'), 1.0)
        tid = INVALID
        if img is not None:
            tid = self.texture(img)
            scale = F(p['scale']) if isinstance(p.get('scale'), (int, float)) else F(1.0)
            avg = (self.tex_avg[tid] * np.array(factor, np.float32)).astype(np.float32)
            L['kind'] = EMIT_RGB
            L['scale'] = scale
            L['coef'] = [factor[0], factor[1], factor[2], 0.0]
            L['rgb_avg'][:3] = (avg * scale).astype(np.float32)
        else:
            self.emitter(p, L)
        o2w = transform(p.get('o2w'))
        L['pos'][:3] = o2w[:3, 3]
        L['dir'][:3] = _normalize(o2w[:3, 2])
        inv = np.linalg.inv(o2w[:3, :3].astype(np.float64))
        w2o = np.zeros((3, 4))
        w2o[:, :3] = inv
        w2o[:, 3] = -inv @ o2w[:3, 3].astype(np.float64)
        ratio = F(p.get('ratio', 1.0))
        if ratio == 0.0:
            W, H = self.textures[tid][1:3] if tid != INVALID else (1, 1)
            ratio = F(F(W) / F(H))
        angle = F(F(min(max(F(p.get('angle', 45.0)), F(1.0)), F(89.0))) * F(PI / F(180.0)))
        tan_y = F(math.tan(angle))
        block = np.zeros(16, np.float32)
        block[:12] = w2o.astype(np.float32).ravel()
        block[12], block[13] = F(ratio * tan_y), tan_y
        block[14] = np.array([tid], np.uint32).view(np.float32)[0]
        L['alias_offset'] = self.spd_len
        self.spd.append(block)
        self.spd_len += 16
        # Projector::power (projector.cpp:60-90).
        y = F(math.sqrt(F(F(1.0) / F(F(ratio * ratio) + F(1.0)))))
        x = F(ratio * y)
        z = F(math.sqrt(F(F(x * x) + F(y * y))))
        p0, p1, p2 = (np.array(v, np.float64) for v in ((x, y, z), (x, -y, z), (-x, -y, z)))
        crosses = []
        for a, b in ((p0, p1), (p1, p2), (p2, p0)):
            c = np.cross(a, b)
            crosses.append(c / np.linalg.norm(c) if np.dot(c, c) > 0 else c)
        c01, c12, c20 = crosses
        solid = abs(math.acos(np.clip(np.dot(c01, -c12), -1, 1)) + math.acos(np.clip(np.dot(c12, -c20), -1, 1)) +
                    math.acos(np.clip(np.dot(c20, -c01), -1, 1)) - math.pi)
        L['lum_power'] = luminance(L['rgb_avg'][:3] * F(F(2.0 * solid) / F(4.0 * PI)))
        self.lights.append(L)

    def sky(self, p):
        """The procedural `sky` node: a lat-long image (row 0 at the zenith)
        with a horizon-to-zenith gradient (sqrt of the elevation fraction),
        a flat ground colour below the horizon and a sun lobe of sun_radius
        degrees, raised-cosine shaped with peak sun_peak."""
        W, H = int(p.get('width', 2048)), int(p.get('height', 1024))
        zen, hor, gnd = (_f3(p.get(k), d) for k, d in (('zenith', (0.25, 0.45, 1.0)),
                                                          ('horizon', (1.0, 0.95, 0.85)),
                                                          ('ground', (0.3, 0.28, 0.25))))
        elev = float(p.get('sun_elevation', 35.0)) * math.pi / 180.0
        azim = float(p.get('sun_azimuth', 40.0)) * math.pi / 180.0
        rad = float(p.get('sun_radius', 5.0)) * math.pi / 180.0
        peak = float(p.get('sun_peak', 5e4))
        sun = np.array([math.cos(elev) * math.cos(azim), math.cos(elev) * math.sin(azim), math.sin(elev)])
        theta = (np.arange(H) + 0.5) / H * math.pi
        phi = (np.arange(W) + 0.5) / W * 2.0 * math.pi
        th, ph = np.meshgrid(theta, phi, indexing='ij')
        d = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
        e = 0.5 * math.pi - th
        t = np.sqrt(np.maximum(e, 0.0) / (0.5 * math.pi))
        c = np.where((e >= 0.0)[..., None], hor + (zen - hor) * t[..., None], gnd)
        ang = np.arccos(np.clip(d @ sun, -1.0, 1.0))
        c = c + np.where(ang < rad, peak * 0.5 * (1.0 + np.cos(math.pi * ang / max(rad, 1e-30))), 0.0)[..., None]
        tex = np.zeros((H, W, 4), np.float32)
        tex[..., :3] = c
        return tex, W, H

    def spherical(self, p, world_lo, world_hi):
        """SphericalMap (spherical.cpp:26-215) over the procedural sky with its
        AliasTable2D (alias2d.cpp:30-66) from luminance * sin(theta) weights
        (calculate_weights, spherical.cpp:150-185)."""
        node = _node(p.get('color'))
        kind = _node_type(node)
        if kind not in ('sky', 'image'):
            raise Unsupported('spherical light colour other than an image or the procedural sky')
        if kind == 'sky':
            tex, W, H = self.sky(node.get('param', {}))
        else:
            tex = load_texels(node, self.base_dir)
            H, W = tex.shape[:2]
        env = np.zeros(1, ENV)[0]
        env['width'], env['height'] = W, H
        env['scale'] = F(p['scale']) if isinstance(p.get('scale'), (int, float)) else F(1.0)
        o2w = transform(p.get('o2w'))
        flip = bool(p.get('flip_u', False))
        rx = _mat_mul(_rot((1, 0, 0), -90.0), _scale((1.0, 1.0 if flip else -1.0, 1.0)))
        o2w = _mat_mul(o2w, rx)
        env['o2w'] = o2w.T.ravel()
        w2o = np.eye(4)
        inv = np.linalg.inv(o2w[:3, :3].astype(np.float64))
        w2o[:3, :3] = inv
        w2o[:3, 3] = -inv @ o2w[:3, 3].astype(np.float64)
        env['w2o'] = w2o.astype(np.float32).T.ravel()
        idx = np.arange(W * H)
        # The reference's per-texel row position: idx / res.y + 0.5 over res.x.
        v = (idx // H).astype(np.float32) + F(0.5)
        sin_t = np.sin((PI * (v / F(W))).astype(np.float64)).astype(np.float32)
        flat = tex.reshape(-1, 4)
        lum = ((F(0.212671) * flat[:, 0] + F(0.715160) * flat[:, 1]) + F(0.072169) * flat[:, 2]).astype(np.float32)
        weights = (lum * sin_t).astype(np.float32)
        cond, cond_func, marg = [], [], np.zeros(H, np.float32)
        for r in range(H):
            row = weights[r * W:(r + 1) * W]
            tab, _, integral = alias_build(row)
            marg[r] = integral
            cond.append(tab)
            cond_func.append(row)
        mtab, _, integral = alias_build(marg)
        env['integral'] = integral
        radius = max(F(F(0.5) * F(np.linalg.norm((world_hi - world_lo).astype(np.float64)))),
                     F(self.doc.get('render_setting', {}).get('min_world_radius', 10.0)))
        env['world_diameter'] = F(F(2.0) * radius)
        a = (flat[:, :3].astype(np.float64).mean(0) * float(env['scale'])).astype(np.float32)
        env['lum_power'] = luminance(a * F(PI * F(radius * radius)))
        self.env = dict(env=env, env_tex=tex.reshape(-1), env_marginal=mtab, env_marginal_func=marg,
                        env_cond=np.concatenate(cond), env_cond_func=np.concatenate(cond_func))
        self.env_power = env['lum_power']

    def camera(self, cj):
        """Sensor (sensor.cpp:20-83,163-172): fov clamped to [15, 120]; the
        transform's pitch and yaw rebuild c2w = T * scale(1, 1, -1) * Ry(yaw) *
        Rx(-pitch); the screen window of the film's aspect ratio
        (radiance_collector.cpp:33-42); filter and lens settings."""
        t = cj.get('type', 'pinhole')
        if t not in ('pinhole', 'thin_lens'):
            raise Unsupported('camera ' + t)
        p = cj.get('param', {})
        cam = np.zeros(1, CAMERA)[0]
        fov = min(max(F(p.get('fov_y', 20.0)), F(15.0)), F(120.0))
        m = transform(p.get('transform'))
        pitch = F(F(math.atan2(m[2, 1], m[1, 1])) * F(180.0) / PI)
        yaw = F(F(math.atan2(m[0, 2], m[0, 0])) * F(180.0) / PI)
        c2w = _mat_mul(_mat_mul(_translate(m[:3, 3]), _scale((1, 1, -1))), _rot((0, 1, 0), yaw))
        c2w = _mat_mul(c2w, _rot((1, 0, 0), F(-pitch)))
        cam['c2w'] = c2w.T.ravel()
        cam['tan_half_fov'] = F(math.tan(F(F(fov * PI / F(180.0)) * F(0.5))))
        rc = p.get('radiance_collector', {}).get('param', {})
        res = rc.get('resolution', [1280, 720])
        w, h = int(res[0]), int(res[1])
        cam['width'], cam['height'] = w, h
        ratio = F(F(w) / F(h))
        lo_x, hi_x, lo_y, hi_y = F(-1), F(1), F(-1), F(1)
        if ratio > 1:
            lo_x, hi_x = -ratio, ratio
        else:
            lo_y, hi_y = F(F(-1) / ratio), F(F(1) / ratio)
        cam['screen_lo_x'], cam['screen_hi_y'] = lo_x, hi_y
        cam['screen_span_x'], cam['screen_span_y'] = F(hi_x - lo_x), F(hi_y - lo_y)
        cam['exposure'] = F(rc.get('exposure', 1.0))
        cam['thin_lens'] = 1 if t == 'thin_lens' else 0
        cam['lens_radius'] = F(p.get('lens_radius', 0.0))
        cam['focal_distance'] = F(p.get('focal_distance', 5.0))
        fj = p.get('filter', {}) or {}
        ft = fj.get('type', 'box')
        if ft not in FILTERS:
            raise Unsupported('filter ' + ft)
        fp = fj.get('param', {}) or {}
        rad = fp.get('radius', [0.5, 0.5])
        rad = rad if isinstance(rad, list) else [rad]
        cam['filter_rx'] = F(rad[0]) if rad else F(0.5)
        cam['filter_ry'] = F(rad[1]) if len(rad) > 1 else cam['filter_rx']
        cam['filter'] = FILTERS[ft]
        if ft == 'gaussian':
            cam['filter_p0'] = F(fp.get('sigma', 1.0))
        elif ft == 'mitchell':
            cam['filter_p0'], cam['filter_p1'] = F(fp.get('b', 1.0 / 3.0)), F(fp.get('c', 1.0 / 3.0))
        elif ft == 'sinc':
            cam['filter_p0'] = F(fp.get('tau', 3.0))
        return cam

    def build(self):
        doc = self.doc
        sp = doc.get('spectrum', {}) or {}
        stype = sp.get('type', 'srgb')
        if stype == 'srgb':
            self.srgb, dim = True, 3
        elif stype == 'hero':
            self.srgb, dim = False, int(sp.get('param', {}).get('dimension', 3))
        else:
            raise Unsupported('spectrum ' + stype)
        for m in doc.get('materials', []):
            self.material(m)
        for sh in doc.get('shapes', []):
            self.shape(sh)
        pos = np.concatenate(self.pos).astype(np.float32)
        ls = doc.get('light_sampler', {}) or {}
        self.env = None
        self.env_power = None
        for l in (ls.get('param', {}) or {}).get('lights', []):
            lt = l.get('type', 'area')
            if lt in ('point', 'spot'):
                self.point_light(lt, l.get('param', {}))
            elif lt == 'projector':
                self.projector(l.get('param', {}))
            elif lt == 'spherical':
                if self.env is not None:
                    raise Unsupported('two environment lights')
                self.spherical(l.get('param', {}), pos.min(0), pos.max(0))
            else:
                raise Unsupported('light ' + lt)
        weights = [L['lum_power'] for L in self.lights] + ([self.env_power] if self.env is not None else [])
        if not weights:
            raise Unsupported('scene without lights')
        light_alias, light_pmf, _ = alias_build(weights)
        ij = doc.get('integrator', {}) or {}
        if ij.get('type', 'pt') != 'pt':
            raise Unsupported('integrator ' + ij.get('type'))
        ipar = ij.get('param', {}) or {}
        ip = np.zeros(1, INTEGRATOR)[0]
        ip['max_depth'] = int(ipar.get('max_depth', 16))
        ip['min_depth'] = int(ipar.get('min_depth', 5))
        ip['rr_threshold'] = F(ipar.get('rr_threshold', 1.0))
        ip['mis_mode'] = int(ipar.get('mis_mode', 0))
        ip['spectrum_dim'] = dim
        disp = any(m['flags'] & FLAG_DISPERSIVE for m in self.materials)
        ip['scatter_pdf_dim'] = dim if disp and not self.srgb else 1
        smp = doc.get('sampler', {}) or {}
        ip['sampler'] = {'independent': 0, 'pcg': 1}[smp.get('type', 'independent')]
        ip['seed'] = int((smp.get('param', {}) or {}).get('seed', 0))
        ip['light_sampler'] = {'uniform': 0, 'power': 1}[ls.get('type', 'uniform')]
        ip['light_count'] = len(weights)
        ip['srgb'] = 1 if self.srgb else 0
        cam = self.camera(doc.get('camera', {}) or {})
        arr = dict(pos=pos.ravel(), nrm=np.concatenate(self.nrm).astype(np.float32).ravel(),
                   uv=np.concatenate(self.uv).astype(np.float32).ravel(),
                   idx=np.concatenate(self.idx).astype(np.uint32), prim_inst=np.concatenate(self.prim_inst),
                   instances=np.array(self.instances, INSTANCE), materials=np.array(self.materials, MATERIAL),
                   lights=np.array(self.lights, LIGHT),
                   prim_alias=np.concatenate(self.prim_alias) if self.prim_alias else np.zeros(0, ALIAS),
                   prim_pmf=(np.concatenate(self.prim_pmf) if self.prim_pmf else np.zeros(0, np.float32)),
                   light_alias=light_alias, light_pmf=light_pmf, camera=np.array([cam], CAMERA),
                   integrator=np.array([ip], INTEGRATOR),
                   spd=np.concatenate(self.spd) if self.spd else np.zeros(0, np.float32))
        if self.env is not None:
            arr.update(self.env)
            arr['env'] = np.array([self.env['env']], ENV)
            arr['rgb2spec'] = np.ascontiguousarray(rgb2spec_table()).reshape(-1)
        if self.textures:
            arr['tex_texels'] = np.concatenate(self.tex_texels).astype(np.float32)
            arr['textures'] = np.array(self.textures, np.uint32).ravel()
            arr['rgb2spec'] = np.ascontiguousarray(rgb2spec_table()).reshape(-1)
        info = dict(vertex_count=self.nverts, prim_count=self.nprims, instance_count=len(self.instances),
                    material_count=len(self.materials), light_count=len(self.lights),
                    width=int(cam['width']), height=int(cam['height']))
        return arr, info


def build(doc, base_dir='.'):
    """Flat arrays (VS_EXPORT_* layout) and counts of a vision_scene.json
    document (a dict or JSON text)."""
    if isinstance(doc, str):
        doc = json.loads(doc)
    return _Builder(doc, base_dir).build()
