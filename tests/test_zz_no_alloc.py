"""vs_render_noalloc — the render entry point for callers that cannot allocate
device memory at render time (a frame loop inside a fixed memory budget, or an
application whose own allocator owns the device memory).  It must give the
same film as vs_render, over two calls in a row that continue one film, and
refuse resolutions beyond its fixed scratch.  Kept in the last-collected file
so that a stop-at-first-failure run has already run every other test."""
import ctypes

import numpy as np
import pytest

from vision_b200 import scenes

pytestmark = pytest.mark.gpu


def test_noalloc_matches_render_over_two_calls(vb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    ctx = vb.Context(0)
    s = vb.Scene(ctx, scenes.box_room(width=64, height=48)).build_accel()
    # Reference films from the allocating entry point.
    s.render(0, 5)
    ref5 = s.film()
    s.render(0, 8)
    ref8 = s.film()

    film = torch.zeros((48, 64, 4), dtype=torch.float32, device='cuda')
    ptr = ctypes.c_void_p(film.data_ptr())
    rc = vb.lib.vs_render_noalloc(s.handle, 0, 5, ptr, None)
    assert rc == vb.VS_OK, vb.lib.vs_last_error(ctx.handle)
    s.synchronize()
    got5 = film.cpu().numpy()
    np.testing.assert_allclose(got5, ref5, rtol=1e-6, atol=1e-7)
    rc = vb.lib.vs_render_noalloc(s.handle, 5, 3, ptr, None)
    assert rc == vb.VS_OK, vb.lib.vs_last_error(ctx.handle)
    s.synchronize()
    got8 = film.cpu().numpy()
    np.testing.assert_allclose(got8, ref8, rtol=1e-6, atol=1e-7)
    assert np.isfinite(got8).all() and got8[..., :3].mean() > 0.0


def test_noalloc_rejects_resolution_beyond_scratch(vb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    ctx = vb.Context(0)
    s = vb.Scene(ctx, scenes.box_room(width=16, height=16)).build_accel()
    s.set_resolution(2048, 1024)
    film = torch.zeros((1024, 2048, 4), dtype=torch.float32, device='cuda')
    rc = vb.lib.vs_render_noalloc(s.handle, 0, 1, ctypes.c_void_p(film.data_ptr()), None)
    assert rc == vb.VS_E_RANGE
    assert '1048576' in vb.lib.vs_last_error(ctx.handle).decode()


def test_noalloc_rejects_misaligned_film(vb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    ctx = vb.Context(0)
    s = vb.Scene(ctx, scenes.box_room(width=16, height=16)).build_accel()
    film = torch.zeros((16 * 16 + 1) * 4, dtype=torch.float32, device='cuda')
    n0 = vb.launch_count()
    rc = vb.lib.vs_render_noalloc(s.handle, 0, 1, ctypes.c_void_p(film.data_ptr() + 4), None)
    assert rc == vb.VS_E_INVALID
    assert 'aligned' in vb.lib.vs_last_error(ctx.handle).decode()
    assert vb.launch_count() == n0, 'a kernel was launched for a rejected call'
