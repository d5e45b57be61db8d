"""The SDK's geometry entry points (reference VisionRenderer::add_instance,
clear_geometries, invalidation; src/sdk/vision.h:66-80, vision.cpp:104-188)
through the C ABI: a scene assembled through add_instance equals the same
scene loaded from JSON, and a C++ host compiled against include/vision_b200.h
drives the library."""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import scene as oscene
from vision_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _split_box_room(**kw):
    """The box room from JSON, and the same room without its two boxes plus
    the boxes' meshes, transforms and materials for add_instance (the JSON
    twin lists the boxes last, in the order they are added)."""
    full = scenes.box_room(**kw)
    boxes = [s for s in full['shapes'] if s['type'] == 'cube']
    rest = [s for s in full['shapes'] if s['type'] != 'cube']
    json_twin = dict(full, shapes=rest + boxes)
    sdk_base = dict(full, shapes=rest)
    adds = []
    for b in boxes:
        P, N, UV, idx = oscene.cube(b['param'])
        m = np.array(b['param']['transform']['param']['matrix4x4'], np.float32).T
        adds.append((P, idx.reshape(-1, 3), N, UV, m, b['param']['material']))
    return json_twin, sdk_base, adds


def test_add_instance_equals_json_scene(vb, host_ctx):
    json_twin, sdk_base, adds = _split_box_room(width=32, height=32)
    a = vb.Scene(host_ctx, json_twin).build_accel()
    b = vb.Scene(host_ctx, sdk_base)
    ids = [b.add_instance(P, t, normals=N, uvs=UV, o2w=m, material=mat) for P, t, N, UV, m, mat in adds]
    assert ids == [6, 7]  # after the five walls and the light
    b.build_accel()
    for k in ('pos', 'nrm', 'uv', 'idx', 'prim_inst', 'instances', 'materials', 'lights', 'light_alias', 'light_pmf',
              'prim_alias', 'camera', 'integrator'):
        assert np.array_equal(a.export(k), b.export(k)), k


def test_add_instance_material_node_and_default(vb, host_ctx):
    sc = scenes.box_room(width=16, height=16)
    s = vb.Scene(host_ctx, sc)
    n0 = s.info()['material_count']
    P, N, UV, idx = oscene.cube({'x': 0.2, 'y': 0.2, 'z': 0.2})
    s.add_instance(P, idx.reshape(-1, 3), material={'type': 'metal', 'param': {'material_name': 'Au',
                                                                              'roughness': 0.3}})
    s.add_instance(P, idx.reshape(-1, 3), o2w=np.diag([1.0, 2.0, 1.0, 1.0]))
    s.build_accel()
    assert s.info()['material_count'] == n0 + 2
    mats = s.export('materials').view(oscene.MATERIAL)
    ref = vb.Scene(host_ctx, scenes.material_room(16, 16)).export('materials').view(oscene.MATERIAL)
    gold = ref[[i for i, m in enumerate(scenes.material_room(16, 16)['materials']) if m['name'] == 'TallBox'][0]]
    assert mats[n0]['type'] == gold['type'] and np.array_equal(mats[n0]['p'], gold['p'])
    assert mats[n0 + 1]['type'] == oscene.DIFFUSE
    pos = s.export('pos', np.float32).reshape(-1, 3)
    assert np.isclose(pos[-24:, 1].max(), 0.2)  # scaled by 2 in y
    with pytest.raises(vb.VisionError) as e:
        s.add_instance(P, idx.reshape(-1, 3), material='NoSuchMaterial')
    assert 'NoSuchMaterial' in str(e.value)
    with pytest.raises(vb.VisionError):
        s.add_instance(P, np.array([[0, 1, 99]]))


def test_clear_geometries_then_rebuild(vb, host_ctx):
    json_twin, sdk_base, adds = _split_box_room(width=16, height=16)
    s = vb.Scene(host_ctx, json_twin).build_accel()
    light = s.export('lights').copy()
    s.clear_geometries()
    info = s.info()
    assert info['prim_count'] == 0 and info['instance_count'] == 0 and info['light_count'] == 0
    assert vb.lib.vs_scene_build_accel(s.handle) == vb.VS_E_STATE
    # Geometry back through add_instance: the walls (no emitter), then the
    # boxes; without an emitter the scene still has no light.
    for P, t, N, UV, m, mat in adds:
        s.add_instance(P, t, normals=N, uvs=UV, o2w=m, material=mat)
    assert vb.lib.vs_scene_build_accel(s.handle) == vb.VS_E_STATE
    assert 'no lights' in vb.lib.vs_last_error(host_ctx.handle).decode()
    assert light.size > 0


def _build_host_program(tmp_path):
    exe = tmp_path / 'sdk_host'
    cmd = ['g++', '-std=c++17', '-O1', '-I', os.path.join(ROOT, 'include'), os.path.join(ROOT, 'tests', 'cpp',
           'sdk_host.cpp'), '-L', os.path.join(ROOT, 'vision_b200'), '-lvision_b200',
           '-Wl,-rpath,' + os.path.join(ROOT, 'vision_b200'), '-o', str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_host_program_builds_and_runs_host_only(vb, tmp_path):
    exe = _build_host_program(tmp_path)
    scene = tmp_path / 'scene.json'
    scene.write_text(json.dumps(scenes.box_room(width=32, height=24)))
    out = subprocess.run([str(exe), str(scene), '-1', '1'], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == 'prims=48 instances=9 lights=1 added=8', out.stdout


@pytest.mark.gpu
def test_cpp_host_program_renders(vb, gpu_ctx, tmp_path):
    # The C++ host's film equals the Python binding's render of the same
    # scene (the same box added through the same entry point).
    exe = _build_host_program(tmp_path)
    sc = scenes.box_room(width=32, height=24)
    scene = tmp_path / 'scene.json'
    scene.write_text(json.dumps(sc))
    film_path = tmp_path / 'film.bin'
    subprocess.run([str(exe), str(scene), '0', '4', str(film_path)], check=True)
    got = np.fromfile(film_path, np.float32).reshape(24, 32, 4)
    s = vb.Scene(gpu_ctx, sc)
    h, c, sn = 0.15, 0.95105652, -0.30901699
    corners = np.array([[(h if i & 1 else -h), (h if i & 2 else -h), (h if i & 4 else -h)] for i in range(8)])
    tri = np.array([0, 2, 1, 1, 2, 3, 4, 5, 6, 5, 7, 6, 0, 1, 4, 1, 5, 4, 2, 6, 3, 3, 6, 7, 0, 4, 2, 2, 4, 6,
                    1, 3, 5, 3, 7, 5]).reshape(-1, 3)
    o2w = np.array([[c, 0, sn, 0.17], [0, 1, 0, 0.15], [-sn, 0, c, 0.12], [0, 0, 0, 1]], np.float32)
    s.add_instance(corners, tri, o2w=o2w, material={'type': 'diffuse', 'param': {'color': [0.2, 0.6, 0.3]}})
    s.build_accel()
    for f in range(4):
        s.render(f, 1)
    assert np.array_equal(got, s.film())
    assert got[..., :3].mean() > 0


@pytest.mark.gpu
def test_programmatic_scene_renders_like_json(vb, gpu_ctx):
    json_twin, sdk_base, adds = _split_box_room(width=48, height=40, sampler='pcg')
    a = vb.Scene(gpu_ctx, json_twin).build_accel()
    b = vb.Scene(gpu_ctx, sdk_base)
    for P, t, N, UV, m, mat in adds:
        b.add_instance(P, t, normals=N, uvs=UV, o2w=m, material=mat)
    b.build_accel()
    a.render(0, 8)
    b.render(0, 8)
    assert np.array_equal(a.film(), b.film())


@pytest.mark.gpu
def test_invalidate_restarts_the_film(vb, gpu_ctx):
    s = vb.Scene(gpu_ctx, scenes.box_room(width=16, height=16)).build_accel()
    s.render(0, 4)
    first = s.film()
    s.invalidate()
    assert vb.lib.vs_render(s.handle, 4, 1, 0, None) == vb.VS_E_STATE
    s.render(0, 4)
    assert np.array_equal(first, s.film())
