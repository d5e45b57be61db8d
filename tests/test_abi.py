"""The C-ABI library loads, exports every symbol the header declares and
reports errors through status codes and vs_last_error (no compute calls)."""
import ctypes
import json
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, 'include', 'vision_b200.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(vs_[a-z0-9_]+)\s*\(', text)))


def test_header_symbols_exported(vb):
    lib = ctypes.CDLL(vb.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(syms) == vb.ABI_SYMBOLS


def test_version(vb):
    assert vb.lib.vs_version() == 100


def test_unsupported_plugin_is_reported(vb, host_ctx):
    from vision_b200 import scenes
    sc = scenes.box_room()
    sc['materials'][0]['type'] = 'subsurface'
    with pytest.raises(vb.UnsupportedError) as e:
        vb.Scene(host_ctx, sc)
    assert 'subsurface' in str(e.value)
    assert e.value.code == vb.VS_E_UNSUPPORTED


def test_parse_error_is_reported(vb, host_ctx):
    with pytest.raises(vb.VisionError) as e:
        vb.Scene(host_ctx, '{"shapes": [ {"type": "quad", ')
    assert e.value.code == vb.VS_E_PARSE


def test_unknown_material_reference(vb, host_ctx):
    from vision_b200 import scenes
    sc = scenes.box_room()
    sc['shapes'][0]['param']['material'] = 'Nope'
    with pytest.raises(vb.VisionError) as e:
        vb.Scene(host_ctx, sc)
    assert 'Nope' in str(e.value)


def test_host_context_cannot_render(vb, host_ctx):
    from vision_b200 import scenes
    s = vb.Scene(host_ctx, scenes.box_room(width=8, height=8)).build_accel()
    with pytest.raises(vb.VisionError) as e:
        s.render(0, 1)
    assert e.value.code == vb.VS_E_NO_DEVICE


def test_render_before_build_is_a_state_error(vb, host_ctx):
    from vision_b200 import scenes
    s = vb.Scene(host_ctx, scenes.box_room(width=8, height=8))
    assert s.info()['accel_built'] == 0


def test_comments_and_trailing_commas(vb, host_ctx):
    from vision_b200 import scenes
    text = json.dumps(scenes.box_room(width=8, height=8), indent=1)
    text = text.replace('"shapes": [', '"shapes": [ // box room\n /* block\n comment */', 1)
    text = text.replace('"render_setting"', '"render_setting"', 1)
    text = text[:-1].rstrip() + ',\n}'
    s = vb.Scene(host_ctx, text)
    assert s.info()['prim_count'] == 36


def test_server_needs_device(vb, host_ctx):
    with pytest.raises(vb.VisionError):
        vb.Server(host_ctx)
