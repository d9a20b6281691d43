"""The render entry point that allocates nothing (gyt_render_device_noalloc).

Some callers cannot allocate GPU memory while they render: engines that own
all device memory through their own allocator or a fixed budget, and code
that runs where cudaMalloc is not allowed. This entry point keeps its paths in
flight in a scratch array built into the library. Here it is called through
the C ABI twice in a row and must give the film of the allocating entry point
(gyt_render_device) up to the summation order of the FP64 film atomics.

This file is collected last so that a failure here does not hide the others.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _film(ctx, scene, sd, fn):
    import torch
    film = torch.zeros(sd.camera.res_x * sd.camera.res_y * 4, dtype=torch.float64, device="cuda")
    fn(film.data_ptr())
    torch.cuda.synchronize()
    return film.cpu().numpy().reshape(sd.camera.res_y, sd.camera.res_x, 4)


def test_noalloc_matches_allocating_render_twice():
    import torch
    import gyunity_b200 as g
    from gyunity_b200 import scenes, _capi

    torch.cuda.init()
    ctx = g.Context(0)
    sd = scenes.mixed_materials_box(level=3, res=96, spp=8)
    scene = g.Scene(sd, ctx)
    want = _film(ctx, scene, sd, lambda p: ctx.render_device(scene, sd.camera, sd.params, p))
    for call in range(2):  # the scratch array keeps the previous call's contents
        got = _film(ctx, scene, sd, lambda p: ctx.check(ctx.render_device_noalloc(scene, sd.camera, sd.params, p)))
        assert np.array_equal(got[..., 3], want[..., 3]), call  # same samples per pixel
        assert np.allclose(got[..., :3], want[..., :3], rtol=1e-9, atol=1e-12), call
    # a pool smaller than the image still covers every sample
    got = _film(ctx, scene, sd, lambda p: ctx.check(ctx.render_device_noalloc(scene, sd.camera, sd.params, p, 1000)))
    assert np.allclose(got[..., :3], want[..., :3], rtol=1e-9, atol=1e-12)
    # sizes beyond the built-in array are rejected with a status and a message
    import ctypes
    rc = ctx.render_device_noalloc(scene, sd.camera, sd.params, 0, _capi.NOALLOC_MAX_PATHS + 1)
    assert rc != 0
    film = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = ctx.render_device_noalloc(scene, sd.camera, sd.params, film.data_ptr(), _capi.NOALLOC_MAX_PATHS + 1)
    assert rc == 4 and b"scratch" in ctx._lib.gyt_last_error(ctx.handle)
    # a pool far too small for the render (a 1024x1024, 16 spp film one path
    # at a time) is refused before any work, with its reason
    big = scenes.mixed_materials_box(level=3, res=1024, spp=16)
    rc = ctx.render_device_noalloc(scene, big.camera, big.params, film.data_ptr(), 1)
    assert rc == 4 and b"too small" in ctx._lib.gyt_last_error(ctx.handle)
    scene.close()
    ctx.close()


def test_noalloc_allocates_no_device_memory_on_a_fresh_context():
    """On a context that has never rendered (its path pools are not
    allocated), a render through the entry point leaves the device's free
    memory unchanged."""
    import torch
    import gyunity_b200 as g
    from gyunity_b200 import scenes

    torch.cuda.init()
    ctx = g.Context(0)
    sd = scenes.mixed_materials_box(level=3, res=64, spp=4)
    scene = g.Scene(sd, ctx)
    film = torch.zeros(64 * 64 * 4, dtype=torch.float64, device="cuda")
    ctx.check(ctx.render_device_noalloc(scene, sd.camera, sd.params, film.data_ptr()))  # looks up the array
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    ctx.check(ctx.render_device_noalloc(scene, sd.camera, sd.params, film.data_ptr()))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # both calls rendered every sample (a sample on a pixel edge also weighs on the neighbour)
    assert film.view(-1, 4)[:, 3].sum().item() >= 2 * 64 * 64 * 4
    scene.close()
    ctx.close()
