"""The `image` shader node on the host (no GPU): the library's PNG, JPEG and
Radiance HDR decoders against OpenCV / Pillow, the texture records and
colour-slot encoding of the scene loader, the oracle's own ingestion of the
same documents, and the refusals."""
import os

import numpy as np
import pytest

from vision_b200 import scenes
from helpers import write_room_textures

cv2 = pytest.importorskip('cv2')


def _scene_with(vb, ctx, folder, node, slot='color', material='diffuse'):
    sc = scenes.box_room(width=8, height=8)
    mats = {m['name']: m for m in sc['materials']}
    mats['BackWall'].update({'type': material, 'param': {slot: node}})
    return vb.Scene(ctx, sc, base_dir=str(folder))


def _texels(vb, ctx, folder, fn, **kw):
    s = _scene_with(vb, ctx, folder, {'type': 'image', 'param': dict(fn=fn, **kw)})
    rec = s.export('textures', np.uint32).reshape(-1, 4)
    assert rec.shape[0] == 1 and rec[0, 0] == 0
    w, h = int(rec[0, 1]), int(rec[0, 2])
    return s.export('tex_texels', np.float32).reshape(h, w, 4)


def _rgb(img):
    """OpenCV's decode as float RGB in [0, 1] (grey replicated, alpha dropped)."""
    f = img.astype(np.float32) / (65535.0 if img.dtype == np.uint16 else 255.0)
    if f.ndim == 2:
        return np.repeat(f[..., None], 3, 2)
    return f[..., 2::-1]


@pytest.mark.parametrize('kind', ['rgb8', 'rgba8', 'grey8', 'grey16', 'rgb16', 'odd'])
def test_png_decoder_matches_opencv(vb, host_ctx, tmp_path, kind):
    rng = np.random.default_rng(hash(kind) % 1000)
    shape = {'rgb8': (17, 23, 3), 'rgba8': (9, 31, 4), 'grey8': (20, 13), 'grey16': (11, 7), 'rgb16': (6, 5, 3),
             'odd': (1, 37, 3)}[kind]
    dt = np.uint16 if kind.endswith('16') else np.uint8
    img = rng.integers(0, np.iinfo(dt).max + 1, shape, dtype=dt)
    if kind == 'rgb8':
        img[:8] = img[:1]  # runs of equal rows exercise the Up and Paeth filters
    cv2.imwrite(str(tmp_path / 'a.png'), img, [cv2.IMWRITE_PNG_COMPRESSION, 9])
    t = _texels(vb, host_ctx, tmp_path, 'a.png', color_space='linear')
    np.testing.assert_array_equal(t[..., :3], _rgb(cv2.imread(str(tmp_path / 'a.png'), cv2.IMREAD_UNCHANGED)))
    assert np.all(t[..., 3] == 0.0)


@pytest.mark.filterwarnings('ignore::UserWarning')
@pytest.mark.parametrize('mode', ['P', 'LA', 'PA'])
def test_png_palette_and_grey_alpha_match_pillow(vb, host_ctx, tmp_path, mode):
    Image = pytest.importorskip('PIL.Image')
    rng = np.random.default_rng(3)
    if mode == 'LA':
        im = Image.fromarray(rng.integers(0, 256, (12, 10, 2), dtype=np.uint8), 'LA')
        ref = np.repeat(np.asarray(im)[..., :1].astype(np.float32) / 255.0, 3, 2)
    else:
        rgb = Image.fromarray(rng.integers(0, 256, (15, 14, 3), dtype=np.uint8), 'RGB')
        im = rgb.quantize(colors=16)
        if mode == 'PA':
            im.info['transparency'] = bytes(range(0, 256, 16))
        ref = np.asarray(im.convert('RGB')).astype(np.float32) / 255.0
    im.save(str(tmp_path / 'p.png'), **({'transparency': bytes(range(0, 256, 16))} if mode == 'PA' else {}))
    t = _texels(vb, host_ctx, tmp_path, 'p.png', color_space='linear')
    np.testing.assert_array_equal(t[..., :3], ref)


@pytest.mark.parametrize('sampling, grey, rst', [(0x221111, False, 0), (0x111111, False, 0), (0x211111, False, 0),
                                                 (0x221111, True, 0), (0x221111, False, 2)])
def test_jpeg_decoder_within_levels_of_opencv(vb, host_ctx, tmp_path, sampling, grey, rst):
    # Baseline JPEG: the library's float IDCT and centred linear chroma
    # upsampling against libjpeg's integer IDCT and its own upsampling; the
    # two decoders differ by a few 8-bit levels at most.
    y, x = np.mgrid[0:45, 0:61] / 9.0
    img = np.stack([128 + 100 * np.sin(x + 0.3 * y), 128 + 90 * np.cos(0.7 * x - y), 128 + 80 * np.sin(x * y / 3)],
                   -1).astype(np.uint8)
    if grey:
        img = img[..., 0]
    params = [cv2.IMWRITE_JPEG_QUALITY, 92, cv2.IMWRITE_JPEG_SAMPLING_FACTOR, sampling]
    if rst:
        params += [cv2.IMWRITE_JPEG_RST_INTERVAL, rst]
    cv2.imwrite(str(tmp_path / 'a.jpg'), img, params)
    t = _texels(vb, host_ctx, tmp_path, 'a.jpg', color_space='linear')
    ref = _rgb(cv2.imread(str(tmp_path / 'a.jpg'), cv2.IMREAD_UNCHANGED))
    d = np.abs(t[..., :3] - ref) * 255.0
    assert d.max() <= 6.0 and d.mean() <= 0.75


def test_progressive_jpeg_is_refused(vb, host_ctx, tmp_path):
    img = np.full((16, 16, 3), 90, np.uint8)
    cv2.imwrite(str(tmp_path / 'p.jpg'), img, [cv2.IMWRITE_JPEG_PROGRESSIVE, 1])
    with pytest.raises(vb.VisionError, match='progressive'):
        _texels(vb, host_ctx, tmp_path, 'p.jpg')


def test_radiance_hdr_matches_opencv(vb, host_ctx, tmp_path):
    rng = np.random.default_rng(5)
    img = (rng.random((19, 33, 3)) * np.array([4.0, 0.5, 40.0])).astype(np.float32)
    img[3, :] = 0.0
    cv2.imwrite(str(tmp_path / 'e.hdr'), img)
    t = _texels(vb, host_ctx, tmp_path, 'e.hdr')  # linear by default
    np.testing.assert_array_equal(t[..., :3], cv2.imread(str(tmp_path / 'e.hdr'), cv2.IMREAD_UNCHANGED)[..., ::-1])


def test_srgb_is_the_default_colour_space_of_8_bit_files(vb, host_ctx, tmp_path):
    # ImagePool::load_texture (image_pool.cpp:18-23): "srgb" unless the file
    # is .exr / .hdr or the node names a colour space.
    rng = np.random.default_rng(9)
    img = rng.integers(0, 256, (8, 8, 3), dtype=np.uint8)
    cv2.imwrite(str(tmp_path / 'c.png'), img)
    lin = _texels(vb, host_ctx, tmp_path, 'c.png', color_space='linear')[..., :3]
    srgb = _texels(vb, host_ctx, tmp_path, 'c.png')[..., :3]
    c = lin.astype(np.float64)
    ref = np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    np.testing.assert_allclose(srgb, ref, rtol=2e-6, atol=1e-9)


def test_colour_slot_records(vb, host_ctx, tmp_path):
    # A textured slot: flag 32, the texture id's bits in p[7], the constant
    # factor as RGB in coef; one texture per file and colour space.
    write_room_textures(str(tmp_path))
    from oracle import scene as oscene
    s = vb.Scene(host_ctx, scenes.textured_room(8, 8), base_dir=str(tmp_path))
    mats = s.export('materials', oscene.MATERIAL)
    tex = s.export('textures', np.uint32).reshape(-1, 4)
    assert tex.shape[0] == 4  # gradient (srgb), checker, gradient (linear), photo
    textured = [m for m in mats if m['flags'] & 32]
    assert len(textured) == 4
    ids = sorted(int(np.float32(m['p'][7]).view(np.uint32)) for m in textured)
    assert ids == [0, 1, 2, 3]
    floor = [m for m in textured if not np.allclose(m['coef'][:3], 1.0)]
    assert len(floor) == 1
    np.testing.assert_array_equal(floor[0]['coef'], np.float32([0.8, 0.7, 0.6, 0.0]))
    # The slot's average colour (texture mean times the factor) feeds the
    # radiance cache's material table.
    rgb = s.export('material_rgb', np.float32).reshape(-1, 3)
    t = s.export('tex_texels', np.float32).reshape(-1, 4)
    g = tex[int(np.float32(floor[0]['p'][7]).view(np.uint32))]
    mean = t[g[0]:g[0] + g[1] * g[2], :3].astype(np.float64).mean(0)
    assert np.any(np.all(np.abs(rgb - mean * [0.8, 0.7, 0.6]) < 1e-5, axis=1))


def test_oracle_ingestion_matches_library(vb, host_ctx, tmp_path):
    # The oracle's own reading of the document (OpenCV decoding) against the
    # library's records and texels (PNG files: identical bytes decoded).
    import oracle
    write_room_textures(str(tmp_path))
    doc = scenes.textured_room(16, 16, jpeg=False)
    s = vb.Scene(host_ctx, doc, base_dir=str(tmp_path))
    from oracle import scene as oscene
    arr, _ = oscene.build(doc, str(tmp_path))
    np.testing.assert_array_equal(s.export('textures', np.uint32), arr['textures'])
    np.testing.assert_allclose(s.export('tex_texels', np.float32), arr['tex_texels'], rtol=2e-6, atol=1e-9)
    a, b = s.export('materials', oscene.MATERIAL), arr['materials']
    assert a.shape == b.shape
    for f in ('type', 'flags', 'spd0', 'spd1'):
        np.testing.assert_array_equal(a[f], b[f])
    np.testing.assert_allclose(a['coef'], b['coef'], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(a['p'].view(np.uint32)[:, 7], b['p'].view(np.uint32)[:, 7])
    assert oracle.OracleScene.from_json(doc, str(tmp_path)) is not None


def test_environment_map_from_an_image_file(vb, host_ctx, tmp_path):
    # SphericalMap over an `image` node: the file's texels are the map and
    # the warper is built from them as for the procedural sky.
    from oracle import scene as oscene
    rng = np.random.default_rng(11)
    img = (rng.random((16, 32, 3)) * 3.0).astype(np.float32)
    img[2:4, 5:9] = 50.0
    cv2.imwrite(str(tmp_path / 'sky.hdr'), img)
    doc = scenes.box_room(width=8, height=8)
    doc['light_sampler'] = {'type': 'power', 'param': {'lights': [
        {'type': 'spherical', 'param': {'color': {'channels': 'xyz', 'node': {'type': 'image',
                                                                              'param': {'fn': 'sky.hdr'}}},
                                        'scale': 0.5}}]}}
    s = vb.Scene(host_ctx, doc, base_dir=str(tmp_path))
    arr, _ = oscene.build(doc, str(tmp_path))
    env_tex = s.export('env_tex', np.float32).reshape(16, 32, 4)
    np.testing.assert_array_equal(env_tex[..., :3], cv2.imread(str(tmp_path / 'sky.hdr'), cv2.IMREAD_UNCHANGED)[..., ::-1])
    np.testing.assert_array_equal(s.export('env_tex', np.float32), arr['env_tex'])
    np.testing.assert_allclose(s.export('env_cond_func', np.float32), arr['env_cond_func'], rtol=1e-6)
    np.testing.assert_allclose(s.export('env_marginal_func', np.float32), arr['env_marginal_func'], rtol=1e-5)


@pytest.mark.parametrize('node, what', [
    ({'type': 'image', 'param': {'fn': 'a.tga'}}, 'tga'),
    ({'type': 'multiply', 'param': {'lhs': {'type': 'image', 'param': {'fn': 'checker.png'}},
                                    'rhs': {'type': 'image', 'param': {'fn': 'gradient.png'}}}}, 'multiply'),
    ({'type': 'image', 'param': {'fn': 'checker.png', 'color_space': 'aces'}}, 'colour space'),
])
def test_unsupported_image_slots(vb, host_ctx, tmp_path, node, what):
    write_room_textures(str(tmp_path))
    with pytest.raises(vb.UnsupportedError, match=what):
        _scene_with(vb, host_ctx, tmp_path, node)


def test_image_node_outside_colour_slots_is_unsupported(vb, host_ctx, tmp_path):
    write_room_textures(str(tmp_path))
    sc = scenes.box_room(width=8, height=8)
    mats = {m['name']: m for m in sc['materials']}
    mats['BackWall'].update({'type': 'metal', 'param': {'roughness': {'type': 'image',
                                                                      'param': {'fn': 'gradient.png'}}}})
    with pytest.raises(vb.UnsupportedError, match='image'):
        vb.Scene(host_ctx, sc, base_dir=str(tmp_path))


def test_missing_image_file_is_an_error(vb, host_ctx, tmp_path):
    with pytest.raises(vb.VisionError, match='cannot open'):
        _texels(vb, host_ctx, tmp_path, 'nope.png')


def test_projector_records(vb, host_ctx, tmp_path):
    # Projector (projector.cpp:30-126): a delta-position light (shape 3) at
    # o2w's origin; its SPD-table block holds the world-to-light rows, the
    # half-angle tangents and the texture id; ratio 0 takes the image's
    # aspect; the power follows the reference's frustum formula.
    from oracle import scene as oscene
    write_room_textures(str(tmp_path))
    doc = scenes.projector_room(16, 16)
    s = vb.Scene(host_ctx, doc, base_dir=str(tmp_path))
    lights = s.export('lights', oscene.LIGHT)
    spd = s.export('spd', np.float32)
    assert [int(L['shape']) for L in lights] == [3, 3]
    img, warm = lights
    np.testing.assert_allclose(img['pos'][:3], [0.1, 0.55, 1.2], rtol=1e-6)
    b = spd[img['alias_offset']:img['alias_offset'] + 16]
    w2o = np.eye(4)
    w2o[:3] = b[:12].reshape(3, 4)
    # The light's +z axis points at the target; the origin maps to the position.
    tgt = w2o @ np.array([0.0, 0.5, -0.5, 1.0])
    assert tgt[2] > 0 and abs(tgt[0]) < 1e-5 and abs(tgt[1]) < 1e-5
    np.testing.assert_allclose(w2o @ np.array([0.1, 0.55, 1.2, 1.0]), [0, 0, 0, 1], atol=1e-6)
    tan_y = np.tan(np.float32(14.0) * np.float32(np.pi / 180.0))
    np.testing.assert_allclose(b[13], tan_y, rtol=1e-6)
    np.testing.assert_allclose(b[12], tan_y * 64.0 / 48.0, rtol=1e-6)  # checker.png is 64 x 48
    tex = s.export('textures', np.uint32).reshape(-1, 4)
    assert b[14:15].view(np.uint32)[0] < tex.shape[0]
    wb = spd[warm['alias_offset']:warm['alias_offset'] + 16]
    assert wb[14:15].view(np.uint32)[0] == 0xffffffff
    np.testing.assert_allclose(wb[12] / wb[13], 1.5, rtol=1e-6)
    # The oracle's own ingestion agrees (records, block and power).
    arr, _ = oscene.build(doc, str(tmp_path))
    o = arr['lights']
    for f in ('shape', 'kind', 'alias_offset'):
        np.testing.assert_array_equal(lights[f], o[f])
    for f in ('pos', 'dir', 'coef', 'rgb_avg', 'scale', 'lum_power'):
        np.testing.assert_allclose(lights[f], o[f], rtol=2e-5, atol=1e-6)
    np.testing.assert_allclose(spd, arr['spd'], rtol=2e-6, atol=1e-6)
    np.testing.assert_array_equal(s.export('light_pmf', np.float32) > 0, arr['light_pmf'] > 0)


@pytest.mark.parametrize('compression', [0, 1, 2, 3])
@pytest.mark.parametrize('half', [True, False])
def test_openexr_decoder_matches_opencv(vb, host_ctx, tmp_path, compression, half):
    # OpenEXR scanline files written by OpenEXR through OpenCV: NONE, RLE,
    # ZIPS and ZIP, HALF and FLOAT channels; a ragged last ZIP block (37
    # lines), grey (a Y channel) and RGBA; linear by default.
    rng = np.random.default_rng(compression + 10 * half)
    img = (rng.random((37, 29, 3)) * np.array([0.5, 8.0, 300.0])).astype(np.float32)
    img[5:9] = 1.25  # runs for RLE
    params = [cv2.IMWRITE_EXR_COMPRESSION, compression,
              cv2.IMWRITE_EXR_TYPE, cv2.IMWRITE_EXR_TYPE_HALF if half else cv2.IMWRITE_EXR_TYPE_FLOAT]
    cv2.imwrite(str(tmp_path / 'a.exr'), img[..., ::-1], params)
    ref = cv2.imread(str(tmp_path / 'a.exr'), cv2.IMREAD_UNCHANGED)[..., ::-1]
    t = _texels(vb, host_ctx, tmp_path, 'a.exr')
    np.testing.assert_array_equal(t[..., :3], ref)
    if half:
        np.testing.assert_allclose(t[..., :3], img, rtol=1e-3)
    else:
        np.testing.assert_array_equal(t[..., :3], img)
    grey = img[..., 1].copy()
    cv2.imwrite(str(tmp_path / 'g.exr'), grey, params)
    tg = _texels(vb, host_ctx, tmp_path, 'g.exr')
    ref_g = cv2.imread(str(tmp_path / 'g.exr'), cv2.IMREAD_UNCHANGED)
    np.testing.assert_array_equal(tg[..., :3], np.repeat(ref_g[..., None], 3, 2))
    rgba = np.concatenate([img, np.full(img.shape[:2] + (1,), 0.5, np.float32)], -1)
    cv2.imwrite(str(tmp_path / 'c.exr'), rgba[..., [2, 1, 0, 3]], params)
    tc = _texels(vb, host_ctx, tmp_path, 'c.exr')
    np.testing.assert_array_equal(tc[..., :3], cv2.imread(str(tmp_path / 'c.exr'), cv2.IMREAD_UNCHANGED)[..., 2::-1])


def test_openexr_piz_is_unsupported(vb, host_ctx, tmp_path):
    img = np.ones((8, 8, 3), np.float32)
    cv2.imwrite(str(tmp_path / 'p.exr'), img, [cv2.IMWRITE_EXR_COMPRESSION, 4])
    with pytest.raises(vb.UnsupportedError, match='PIZ'):
        _texels(vb, host_ctx, tmp_path, 'p.exr')


REF_SKY = '/root/reference/res/render_scene/cbox/textures/sky.exr'


@pytest.mark.skipif(not os.path.exists(REF_SKY), reason='reference assets absent')
def test_reference_sky_exr_as_environment(vb, host_ctx, tmp_path):
    # The reference's own ZIP / HALF / ABGR map (cbox/textures/sky.exr) as a
    # spherical light: its texels equal OpenEXR's decode.
    sc = scenes.box_room(width=8, height=8)
    sc['light_sampler']['param']['lights'] = [{'type': 'spherical', 'param': {
        'color': {'fn': REF_SKY, 'color_space': 'linear'}, 'scale': 1.0}}]
    s = vb.Scene(host_ctx, sc, base_dir=str(tmp_path))
    env = s.export('env_tex', np.float32).reshape(256, 512, 4)
    ref = cv2.imread(REF_SKY, cv2.IMREAD_UNCHANGED)
    np.testing.assert_array_equal(env[..., :3], ref[..., 2::-1])


@pytest.mark.parametrize('ext', ['png', 'jpg', 'hdr', 'exr'])
def test_corrupt_image_files_fail_cleanly(vb, host_ctx, tmp_path, ext):
    # Truncated and byte-damaged files either decode or raise an error
    # through the C ABI; the decoders check every length, table id, code
    # length and size they read (a damaged JPEG once indexed past its Huffman
    # tables).
    rng = np.random.default_rng(17)
    img = (rng.random((19, 27, 3)) * 255).astype(np.uint8)
    src = tmp_path / ('src.' + ext)
    if ext == 'hdr':
        cv2.imwrite(str(src), img.astype(np.float32) / 7)
    elif ext == 'exr':
        cv2.imwrite(str(src), img.astype(np.float32) / 9, [cv2.IMWRITE_EXR_COMPRESSION, 3])
    elif ext == 'jpg':
        cv2.imwrite(str(src), img, [cv2.IMWRITE_JPEG_RST_INTERVAL, 2])
    else:
        cv2.imwrite(str(src), img)
    raw = src.read_bytes()
    outcomes = set()
    for trial in range(240):
        b = bytearray(raw)
        kind = trial % 3
        if kind == 0:
            b = b[:int(rng.integers(0, len(b)))]
        elif kind == 1:
            for _ in range(int(rng.integers(1, 8))):
                b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
        else:
            i = int(rng.integers(0, len(b)))
            b[i:i + 4] = bytes(rng.integers(0, 256, 4).astype(np.uint8))
        (tmp_path / ('bad.' + ext)).write_bytes(bytes(b))
        try:
            _texels(vb, host_ctx, tmp_path, 'bad.' + ext, color_space='linear')
            outcomes.add('decoded')
        except vb.VisionError:
            outcomes.add('error')
    assert 'error' in outcomes
