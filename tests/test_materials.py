"""Material layer on the host: plugin parameters, SPD slots and the albedo
tables of the compensated lobes (no GPU)."""
import json
import os

import numpy as np
import pytest

from vision_b200 import scenes

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_shipped_albedo_tables_equal_reference(vb):
    g = json.load(open(os.path.join(G, 'albedo_luts.json')))
    t = vb.albedo_luts()
    np.testing.assert_allclose(t[:1024], g['PureReflectionLobe'], rtol=0, atol=1e-6)
    for name, off, ch in (('DielectricLobe', 1024, 2), ('DielectricInvLobe', 1024 + 65536, 2),
                          ('SpecularLobe', 1024 + 131072, 1)):
        for c in g[name]:
            x, y, z = (int(v) for v in c[:3])
            i = off + ((z * 32 + y) * 32 + x) * ch
            np.testing.assert_allclose(t[i:i + ch], c[3:3 + ch], rtol=0, atol=1e-6)


def test_regenerated_albedo_tables_close_to_reference(vb):
    # apps/precompute's job, redone from the lobe definitions.  The shipped
    # values carry the reference's own sampling error (24-bit LCG sample pairs),
    # so agreement is to a few percent, not to float precision.
    g = json.load(open(os.path.join(G, 'albedo_luts.json')))
    t = vb.albedo_luts(regenerated=True)
    d = np.abs(t[:1024] - np.array(g['PureReflectionLobe']))
    assert d.max() < 0.05 and d.mean() < 0.01
    for name, off, ch in (('DielectricLobe', 1024, 2), ('DielectricInvLobe', 1024 + 65536, 2),
                          ('SpecularLobe', 1024 + 131072, 1)):
        diffs = []
        for c in g[name]:
            x, y, z = (int(v) for v in c[:3])
            i = off + ((z * 32 + y) * 32 + x) * ch
            diffs.append(np.abs(t[i:i + ch] - c[3:3 + ch]))
        diffs = np.array(diffs)
        assert diffs.max() < 0.06, name
        assert diffs.mean() < 0.012, name


def test_metal_glass_principled_records(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.material_room(8, 8))
    names = None
    mats = s.export('materials', np.uint32).reshape(-1, 16)
    matf = mats.view(np.float32)
    types = list(mats[:, 0])
    assert types.count(2) == 1 and types.count(3) == 1 and types.count(4) == 1
    metal = matf[types.index(2)]
    # roughness 0.3 remapped to alpha = 0.09 (metal.cpp:143).
    assert abs(metal[8] - 0.09) < 1e-7 and abs(metal[9] - 0.09) < 1e-7
    glass = mats[types.index(3)]
    assert glass[1] & 1  # dispersive: ior is an spd slot
    spd = s.export('spd', np.float32)
    off = glass[2]
    n = int(spd[off])
    assert n == 94
    lam = 360.0 + 5.0 * np.arange(94)
    np.testing.assert_allclose(spd[off + 1:off + 1 + n], 1.5 + 0.0042 / (lam / 1000.0) ** 2, rtol=1e-6)
    info = s.info()
    integ = s.export('integrator', np.uint32)
    assert integ[5] == info['spectrum_dim']  # scatter_pdf_dim = dimension with a dispersive material
    pr = matf[types.index(4)]
    assert abs(pr[8] - 0.35 ** 2) < 1e-6 and abs(pr[10] - 0.4) < 1e-7 and abs(pr[11] - 1.5) < 1e-7


def test_principled_layers_are_recorded(vb, host_ctx):
    # Sheen, coat and transmission parameters (principled_bsdf.cpp:287-302)
    # go to a 12-float block of the SPD table; a principled material without
    # them keeps spd0 unset.
    sc = scenes.principled_room(8, 8)
    s = vb.Scene(host_ctx, sc)
    mats = s.export('materials', np.uint32).reshape(-1, 16)
    names = [m['name'] for m in sc['materials']]
    spd = s.export('spd', np.float32)
    tall = mats[names.index('TallBox')]
    assert tall[0] == 4 and tall[2] != 0xffffffff
    blk = spd[tall[2]:tall[2] + 13]
    assert blk[0] == 12
    np.testing.assert_allclose(blk[[1, 2, 6, 7, 8, 12]], [0.8, 0.4, 0.7, 0.15, 1.6, 0.0], rtol=1e-7)
    short = mats[names.index('ShortBox')]
    blk = spd[short[2]:short[2] + 13]
    np.testing.assert_allclose(blk[[1, 2, 6, 7, 8, 12]], [0.0, 0.5, 0.3, 0.1, 1.5, 0.8], rtol=1e-7)
    plain = vb.Scene(host_ctx, scenes.material_room(8, 8)).export('materials', np.uint32).reshape(-1, 16)
    assert plain[[m['name'] for m in scenes.material_room(8, 8)['materials']].index('Floor')][2] == 0xffffffff


def test_metal_names(vb, host_ctx):
    # The ten conductors of metal_ior.inl.h each get their own (eta, k)
    # table; an unknown name falls back to silver (metal.cpp:104-110).
    def eta_k(name):
        sc = scenes.box_room(width=4, height=4)
        sc['materials'][0] = {'type': 'metal', 'name': 'Floor', 'param': {'material_name': name}}
        s = vb.Scene(host_ctx, sc)
        spd = s.export('spd', np.float32)
        return spd.copy()
    names = ['Ag', 'Al', 'Au', 'Cu', 'CuZn', 'Fe', 'Ti', 'V', 'VN', 'Li']
    tables = {n: eta_k(n) for n in names}
    for i, a in enumerate(names):
        for b in names[i + 1:]:
            assert not np.array_equal(tables[a], tables[b]), (a, b)
    np.testing.assert_array_equal(eta_k('Unobtainium'), tables['Ag'])


def test_mirror_and_substrate_records(vb, host_ctx):
    s = vb.Scene(host_ctx, scenes.substrate_room(8, 8))
    mats = s.export('materials', np.uint32).reshape(-1, 16)
    matf = mats.view(np.float32)
    names = ['Floor', 'Ceiling', 'BackWall', 'LeftWall', 'RightWall', 'TallBox', 'ShortBox', 'Light']
    rec = {n: (mats[i], matf[i]) for i, n in enumerate(names)}
    # Mirror: a metal record with the constant-Fresnel flag, colour
    # coefficients, roughness 0.05 remapped to alpha 0.0025 (mirror.cpp:59-74).
    u, f = rec['TallBox']
    assert u[0] == 2 and (u[1] & 4) and u[2] == 0xffffffff
    assert abs(f[8] - 0.0025) < 1e-9 and abs(f[9] - 0.0025) < 1e-9
    assert np.any(f[4:7] != 0.0)
    # Substrate with remapping squares twice: 0.6 -> 0.36 -> 0.1296
    # (substrate.cpp:133-139); Rs coefficients in p[2..4].
    u, f = rec['ShortBox']
    assert u[0] == 5
    np.testing.assert_allclose(f[8:10], [0.6 ** 4] * 2, rtol=1e-6)
    assert np.any(f[10:13] != 0.0)
    # Unremapped alphas stay as given.
    u, f = rec['Floor']
    assert u[0] == 5
    np.testing.assert_allclose(f[8:10], [0.1, 0.1], rtol=1e-6)
    # Rs defaults to 0.05 grey: the same coefficients as an explicit 0.05.
    sc = scenes.substrate_room(8, 8)
    for m in sc['materials']:
        if m['name'] == 'Floor':
            m['param']['spec'] = [0.05, 0.05, 0.05]
    f2 = vb.Scene(host_ctx, sc).export('materials', np.float32).reshape(-1, 16)[0]
    np.testing.assert_array_equal(f2[10:13], f[10:13])


def test_metallic_records(vb, host_ctx):
    # MetallicMaterial (metallic.cpp:26-60): a metal record with the F82
    # flag, colour coefficients, the edge tint's coefficients in p[2..4],
    # roughness clamped to [0.01, 1] and squared, anisotropy as for metal.
    s = vb.Scene(host_ctx, scenes.metallic_room(8, 8))
    mats = s.export('materials', np.uint32).reshape(-1, 16)
    matf = mats.view(np.float32)
    names = ['Floor', 'Ceiling', 'BackWall', 'LeftWall', 'RightWall', 'TallBox', 'ShortBox', 'Light']
    rec = {n: (mats[i], matf[i]) for i, n in enumerate(names)}
    u, f = rec['TallBox']
    assert u[0] == 2 and (u[1] & 64) and not (u[1] & 4) and u[2] == 0xffffffff
    np.testing.assert_allclose(f[8:10], [0.35 ** 2] * 2, rtol=1e-6)
    assert np.any(f[10:13] != 0.0)
    u, f = rec['ShortBox']
    a = np.float32(0.3) ** 2
    np.testing.assert_allclose(f[8:10], [a * 0.5, a / 0.5], rtol=1e-6)
    # The edge tint defaults to white; roughness below 0.01 clamps.
    sc = scenes.metallic_room(8, 8)
    for m in sc['materials']:
        if m['name'] == 'BackWall':
            m['param'] = {'color': [0.9, 0.9, 0.9], 'edge_tint': [1.0, 1.0, 1.0], 'roughness': 0.001}
    f2 = vb.Scene(host_ctx, sc).export('materials', np.float32).reshape(-1, 16)[2]
    np.testing.assert_array_equal(f2[10:13], rec['BackWall'][1][10:13])
    np.testing.assert_allclose(f2[8:10], [1e-4, 1e-4], rtol=1e-6)


def test_gpu_albedo_tables_need_a_device_and_a_valid_strata(vb, host_ctx):
    with pytest.raises(vb.VisionError) as e:
        vb.albedo_luts_gpu(host_ctx, 32)
    assert e.value.code == vb.VS_E_NO_DEVICE
    with pytest.raises(vb.VisionError) as e:
        vb.albedo_luts_gpu(host_ctx, 0)
    assert e.value.code == vb.VS_E_RANGE


def test_plastic_records(vb, host_ctx):
    # PlasticMaterial (plastic.cpp:80-129): a substrate-class record with the
    # plastic flag, ior in p[5], roughness remapped twice.
    s = vb.Scene(host_ctx, scenes.plastic_room(8, 8))
    mats = s.export('materials', np.uint32).reshape(-1, 16)
    matf = mats.view(np.float32)
    for i, alpha, ior in ((5, 0.1 ** 4, 1.3), (6, 0.3 ** 4, 1.5)):
        assert mats[i, 0] == 5 and (mats[i, 1] & 8)
        np.testing.assert_allclose(matf[i, 8:10], [max(alpha, 1e-4)] * 2, rtol=1e-5)
        np.testing.assert_allclose(matf[i, 13], ior, rtol=1e-6)


def test_mix_and_add_records(vb, host_ctx):
    # MixMaterial / AddMaterial: the inline children become records of their
    # own, in front of the mix record, which holds their indices, the mix
    # fraction and the add flag.
    s = vb.Scene(host_ctx, scenes.mix_room(16, 16))
    from oracle.scene import MATERIAL, MIX, FLAG_ADD, GLASS, DIFFUSE, METAL, PRINCIPLED
    m = s.export('materials').view(MATERIAL)
    mixes = np.nonzero(m['type'] == MIX)[0]
    assert len(mixes) == 4
    kinds = sorted((int(m['type'][m['spd0'][i]]), int(m['type'][m['spd1'][i]]), bool(m['flags'][i] & FLAG_ADD),
                    round(float(m['p'][i][0]), 3)) for i in mixes)
    assert (GLASS, GLASS, False, 0.5) in kinds and (DIFFUSE, METAL, False, 0.3) in kinds
    assert any(k[:3] == (DIFFUSE, PRINCIPLED, True) for k in kinds)
    for i in mixes:
        assert m['spd0'][i] < i and m['spd1'][i] < i


def test_mix_refusals(vb, host_ctx):
    sc = scenes.mix_room(16, 16)
    for mt in sc['materials']:
        if mt['name'] == 'TallBox':
            mt['param']['mat1'] = {'type': 'mix', 'param': {'mat0': {'type': 'diffuse'}, 'mat1': {'type': 'diffuse'}}}
    with pytest.raises(vb.UnsupportedError, match='mix'):
        vb.Scene(host_ctx, sc)
    sc = scenes.mix_room(16, 16, dimension=3)
    sc['integrator'] = {'type': 'rt', 'param': {'max_depth': 4}}
    with pytest.raises(vb.UnsupportedError, match='rt integrator'):
        vb.Scene(host_ctx, sc)
