"""The `model` shape (Model, src/render_core/shapes/model.cpp:27-37; assimp's
OBJ import and post-processing, importers/assimp_parser.cpp:231-340): the
library's loader against a plain-Python restatement of the same rules on
generated Wavefront OBJ files."""
import math

import numpy as np
import pytest

from vision_b200 import scenes

CUBE_OBJ = """# unit cube: quads with v/vt/vn, a triangle fan with v//vn and v only
o cube
v -0.5 -0.5 -0.5
v  0.5 -0.5 -0.5
v  0.5  0.5 -0.5
v -0.5  0.5 -0.5
v -0.5 -0.5  0.5
v  0.5 -0.5  0.5
v  0.5  0.5  0.5
v -0.5  0.5  0.5
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 -1
vn 0 0 1
vn 0 -1 0
vn 0 1 0
g sides
usemtl whatever
f 1/1/1 4/4/1 3/3/1 2/2/1
f 5/1/2 6/2/2 7/3/2 8/4/2
f -8//3 -7//3 -3//3 -4//3
f 4//4 8//4 7//4 3//4
f 1 5 8 4
f 2 3 7
f 2 7 6
"""


def _parse(text, smooth=False, flip_uv=True, swap_handed=False):
    """Plain restatement of the model loader's rules (see the module doc)."""
    P, T, N, corners, tri_face = [], [], [], [], []
    faces = 0
    for raw in text.splitlines():
        tok = raw.split()
        if not tok:
            continue
        if tok[0] == 'v':
            P.append([float(x) for x in tok[1:4]])
        elif tok[0] == 'vt':
            T.append([float(x) for x in tok[1:3]] + [0.0] * (2 - len(tok[1:3])))
        elif tok[0] == 'vn':
            N.append([float(x) for x in tok[1:4]])
        elif tok[0] == 'f':
            poly = []
            for c in tok[1:]:
                parts = c.split('/')
                res = lambda r, n: (int(r) - 1) if int(r) > 0 else n + int(r)
                v = res(parts[0], len(P))
                t = res(parts[1], len(T)) if len(parts) > 1 and parts[1] else -1
                n = res(parts[2], len(N)) if len(parts) > 2 and parts[2] else -1
                poly.append((v, t, n))
            for i in range(1, len(poly) - 1):
                corners += [poly[0], poly[i], poly[i + 1]]
                tri_face.append(faces)
            faces += 1
    P = np.array(P, np.float32)
    N = np.array(N, np.float32).reshape(-1, 3)
    if swap_handed:
        P[:, 2] *= -1
        N[:, 2] *= -1
        for t in range(0, len(corners), 3):
            corners[t + 1], corners[t + 2] = corners[t + 2], corners[t + 1]
    ntri = len(corners) // 3
    tri_n = np.zeros((ntri, 3), np.float32)
    acc = np.zeros_like(P)
    for t in range(ntri):
        k = corners[3 * t:3 * t + 3]
        if all(c[2] >= 0 for c in k):
            continue
        g = np.cross(P[k[1][0]] - P[k[0][0]], P[k[2][0]] - P[k[0][0]])
        l = np.linalg.norm(g)
        tri_n[t] = g / l if l > 0 else 0.0
        for c in k:
            acc[c[0]] += tri_n[t]
    pos, nrm, uv, idx, seen = [], [], [], [], {}
    for t in range(ntri):
        for c in corners[3 * t:3 * t + 3]:
            key = (c[0], c[1], c[2] if c[2] >= 0 else (-1 if smooth else -2 - tri_face[t]))
            if key in seen:
                idx.append(seen[key])
                continue
            seen[key] = len(pos)
            idx.append(len(pos))
            pos.append(P[c[0]])
            if c[2] >= 0:
                n = N[c[2]]
            elif smooth:
                l = np.linalg.norm(acc[c[0]])
                n = acc[c[0]] / l if l > 0 else np.zeros(3, np.float32)
            else:
                n = tri_n[t]
            nrm.append(n)
            u = list(T[c[1]]) if c[1] >= 0 else [0.0, 0.0]
            if c[1] >= 0 and flip_uv:
                u[1] = 1.0 - u[1]
            uv.append(u)
    return (np.array(pos, np.float32), np.array(nrm, np.float32), np.array(uv, np.float32),
            np.array(idx, np.uint32))


def _model_scene(fn, **param):
    sc = scenes.box_room(width=8, height=8)
    sc['shapes'] = [s for s in sc['shapes'] if s['name'] in ('floor', 'light')]
    p = {'fn': fn, 'material': 'TallBox'}
    p.update(param)
    sc['shapes'].append({'type': 'model', 'name': 'model', 'param': p})
    return sc


def _model_arrays(s):
    # The model is the last instance; the floor quad (4 vertices) and the
    # light quad (4) come before it.
    pos = s.export('pos', np.float32).reshape(-1, 3)[8:]
    nrm = s.export('nrm', np.float32).reshape(-1, 3)[8:]
    uv = s.export('uv', np.float32).reshape(-1, 2)[8:]
    idx = s.export('idx', np.uint32)[12:] - 8
    return pos, nrm, uv, idx


@pytest.mark.parametrize('opts', [{}, {'smooth': True}, {'flip_uv': False}, {'swap_handed': True},
                                  {'smooth': True, 'swap_handed': True}])
def test_model_matches_restatement(vb, host_ctx, tmp_path, opts):
    (tmp_path / 'cube.obj').write_text(CUBE_OBJ)
    s = vb.Scene(host_ctx, _model_scene('cube.obj', **opts), base_dir=str(tmp_path))
    pos, nrm, uv, idx = _model_arrays(s)
    e_pos, e_nrm, e_uv, e_idx = _parse(CUBE_OBJ, **opts)
    np.testing.assert_array_equal(idx, e_idx)
    np.testing.assert_allclose(pos, e_pos, atol=1e-7)
    np.testing.assert_allclose(nrm, e_nrm, atol=1e-6)
    np.testing.assert_allclose(uv, e_uv, atol=1e-7)
    # 5 quads (2 triangles each) + 2 triangles: the cube's 12 triangles.
    assert idx.size == 12 * 3


def test_model_transform_and_normals(vb, host_ctx, tmp_path):
    (tmp_path / 'm').mkdir()
    (tmp_path / 'm' / 'tri.obj').write_text('v 0 0 0\nv 1 0 0\nv 0 0 -1\nf 1 2 3\n')
    xf = {'type': 'trs', 'param': {'t': [0.0, 0.25, 0.0], 'r': [0, 1, 0, 0], 's': [2.0, 2.0, 2.0]}}
    s = vb.Scene(host_ctx, _model_scene('m/tri.obj', transform=xf), base_dir=str(tmp_path))
    pos, nrm, _, idx = _model_arrays(s)
    np.testing.assert_allclose(pos, [[0, 0.25, 0], [2, 0.25, 0], [0, 0.25, -2]], atol=1e-6)
    # (p1 - p0) x (p2 - p0) = (1,0,0) x (0,0,-1) = (0, 1, 0).
    np.testing.assert_allclose(nrm / np.linalg.norm(nrm, axis=1, keepdims=True), [[0, 1, 0]] * 3, atol=1e-6)
    assert list(idx) == [0, 1, 2]


def test_trs_transform_rotates_about_the_axis(vb, host_ctx, tmp_path):
    # TransformDesc "trs" (node_desc.cpp:48-52): T * R(axis, degrees) * S.
    (tmp_path / 'tri.obj').write_text('v 0 0 0\nv 1 0 0\nv 0 0 -1\nf 1 2 3\n')
    axis, deg = np.array([1.0, 2.0, 2.0]) / 3.0, 30.0
    xf = {'type': 'trs', 'param': {'t': [0.1, 0.2, 0.3], 'r': [1.0, 2.0, 2.0, deg], 's': [1.0, 2.0, 3.0]}}
    s = vb.Scene(host_ctx, _model_scene('tri.obj', transform=xf), base_dir=str(tmp_path))
    pos = _model_arrays(s)[0]
    a = math.radians(deg)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    R = np.eye(3) + math.sin(a) * K + (1 - math.cos(a)) * K @ K
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 0, -1]], np.float64) * [1.0, 2.0, 3.0]
    np.testing.assert_allclose(pos, P @ R.T + [0.1, 0.2, 0.3], atol=2e-6)


@pytest.mark.parametrize('text, needle', [
    ('v 0 0 0\nv 1 0 0\nf 1 2 3\n', 'index out of range'),
    ('v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1/2 2 3\n', 'index out of range'),
    ('v 0 0\n', '3 coordinates'),
    ('v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 x3\n', 'face corner'),
    ('v 0 0 0\n', 'no faces'),
])
def test_model_rejects_bad_files(vb, host_ctx, tmp_path, text, needle):
    (tmp_path / 'bad.obj').write_text(text)
    with pytest.raises(vb.VisionError, match=needle):
        vb.Scene(host_ctx, _model_scene('bad.obj'), base_dir=str(tmp_path))


def test_model_unsupported_options(vb, host_ctx, tmp_path):
    (tmp_path / 'cube.obj').write_text(CUBE_OBJ)
    with pytest.raises(vb.UnsupportedError, match='subdiv'):
        vb.Scene(host_ctx, _model_scene('cube.obj', subdiv_level=1), base_dir=str(tmp_path))
    with pytest.raises(vb.UnsupportedError, match='obj'):
        vb.Scene(host_ctx, _model_scene('apple.gltf'), base_dir=str(tmp_path))
    with pytest.raises(vb.VisionError, match='cannot open'):
        vb.Scene(host_ctx, _model_scene('missing.obj'), base_dir=str(tmp_path))


def test_model_reader_tolerates_layout_variants(vb, host_ctx, tmp_path):
    # CRLF line ends, tabs, comments, 3-component texture coordinates and a
    # 'w' on positions parse like the plain form.
    plain = 'v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nf 1/1 2/2 3/3 4/4\n'
    variant = ('# quad\r\nv\t0 0 0 1\r\nv 1 0 0 1\r\nv 1 1 0\r\nv 0 1 0\r\n'
               'vt 0 0 0\r\nvt 1 0 0\r\nvt\t1 1 0\r\nvt 0 1 0\r\n\r\ns off\r\nf\t1/1 2/2\t3/3 4/4\r\n')
    out = []
    for name, text in (('plain.obj', plain), ('variant.obj', variant)):
        (tmp_path / name).write_bytes(text.encode())
        s = vb.Scene(host_ctx, _model_scene(name), base_dir=str(tmp_path))
        out.append(_model_arrays(s))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)
