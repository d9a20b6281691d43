"""Batched renders (gyt_render_batch_device): many scenes, cameras and sample
counts in one wavefront must give every instance the film that its own
gyt_render_device call gives (the same paths; FP64 sums in another order).
Needs a B200."""
import dataclasses

import numpy as np
import pytest
import torch

import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu


def _descs():
    a = scenes.cornell_box(res=32, spp=4, max_depth=8, rr_depth=3)
    b = scenes.cornell_box(res=48, spp=2, max_depth=5, rr_depth=1, spheres=False)
    b = dataclasses.replace(b, camera=dataclasses.replace(b.camera, res_x=48, res_y=20))
    c = scenes.procedural_mesh_box(level=4, res=40, spp=3, max_depth=6, rr_depth=2)
    d = scenes.mixed_materials_box(res=24, spp=5)
    e = scenes.env_knot_small()
    return [a, b, c, d, e]


DESCS = _descs()


def _film(cam):
    return torch.zeros(cam.res_x * cam.res_y * 4, dtype=torch.float64, device="cuda")


def _per_scene(ctx, scs, descs):
    films = []
    for sc, sd in zip(scs, descs):
        f = _film(sd.camera)
        ctx.render_device(sc, sd.camera, sd.params, f.data_ptr())
        films.append(f.cpu().numpy())
    return films


def _batch(ctx, scs, descs, order=None):
    order = list(range(len(descs))) if order is None else order
    films = [_film(descs[i].camera) for i in order]
    st = ctx.render_batch_device([scs[i] for i in order], [descs[i].camera for i in order],
                                 [descs[i].params for i in order], [f.data_ptr() for f in films])
    out = [None] * len(descs)
    for k, i in enumerate(order):
        out[i] = films[k].cpu().numpy()
    return out, st


def _same(a, b):
    for fa, fb in zip(a, b):
        np.testing.assert_allclose(fa, fb, rtol=1e-12, atol=1e-12)


@pytest.fixture(scope="module")
def bctx():
    c = g.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def scs(bctx):
    return [g.Scene(sd, bctx) for sd in DESCS]


def test_batch_equals_per_scene(bctx, scs):
    bctx.set_batch_config()
    ref = _per_scene(bctx, scs, DESCS)
    got, st = _batch(bctx, scs, DESCS)
    _same(got, ref)
    assert st["paths"] == sum(sd.n_paths() for sd in DESCS)
    assert st["launches"] > 0 and st["ms"] > 0


def test_batch_refills_across_instances():
    # a pool far smaller than one instance: every refill mixes instances
    c = g.Context(0)
    try:
        scs = [g.Scene(sd, c) for sd in DESCS]
        c.set_batch_config(paths_in_flight=2048)
        got, st = _batch(c, scs, DESCS, order=[4, 2, 0, 3, 1])
        _same(got, _per_scene(c, scs, DESCS))
        assert st["iterations"] > 10
    finally:
        c.close()


def test_batch_graph_and_host_loop_agree(bctx, scs):
    bctx.set_batch_config(use_graph=False)
    try:
        a, sa = _batch(bctx, scs, DESCS)
    finally:
        bctx.set_batch_config()
    b, sb = _batch(bctx, scs, DESCS)
    c, _ = _batch(bctx, scs, DESCS)  # the captured graph again
    _same(a, b)
    _same(b, c)
    assert sa["paths"] == sb["paths"]


def test_batch_host_images(bctx, scs):
    imgs = bctx.render_batch(scs, [sd.camera for sd in DESCS], [sd.params for sd in DESCS])
    for sc, sd, im in zip(scs, DESCS, imgs):
        cam = g.PinHoleCamera(g.Film(sd.camera.res_x, sd.camera.res_y), sd.camera.pos, sd.camera.look_at,
                              sd.camera.up, sd.camera.fovy, sd.camera.film_distance)
        ref = g.GpuPathTracing(sd.params.spp, sd.params.max_depth, sd.params.rr_depth).Render(sc, cam).GetImage()
        np.testing.assert_allclose(im, ref, rtol=1e-6, atol=1e-7)
    # again into caller-owned images (the context's film buffers reused and re-zeroed)
    out = [np.full((sd.camera.res_y, sd.camera.res_x, 3), -1.0, np.float32) for sd in DESCS]
    again = bctx.render_batch(scs, [sd.camera for sd in DESCS], [sd.params for sd in DESCS], out=out)
    for im, o, a in zip(imgs, out, again):
        assert a is o
        np.testing.assert_allclose(o, im, rtol=1e-6, atol=1e-7)
    with pytest.raises(ValueError):
        bctx.render_batch(scs, [sd.camera for sd in DESCS], [sd.params for sd in DESCS], out=out[:-1])


def test_batch_many_small_instances(bctx):
    descs = [scenes.cornell_box(res=8 + 4 * (k % 5), spp=1 + k % 7, max_depth=2 + k % 6, spheres=bool(k % 2))
             for k in range(40)]
    scs = [g.Scene(sd, bctx) for sd in descs]
    got, _ = _batch(bctx, scs, descs)
    _same(got, _per_scene(bctx, scs, descs))


def test_batch_empty_and_invalid(bctx, scs):
    st = bctx.render_batch_device([], [], [], [])
    assert st["paths"] == 0
    with pytest.raises(g.GytError):
        bctx.render_batch_device([scs[0]], [DESCS[0].camera], [DESCS[0].params], [0])
    c8 = g.Context(0, bvh_width=8)
    try:
        w8 = g.Scene(DESCS[0], c8)
        films = [_film(DESCS[0].camera), _film(DESCS[1].camera)]
        with pytest.raises(g.GytError):
            bctx.render_batch_device([w8, scs[1]], [DESCS[0].camera, DESCS[1].camera],
                                     [DESCS[0].params, DESCS[1].params], [f.data_ptr() for f in films])
    finally:
        c8.close()


def test_batch_autotune(bctx, scs):
    cfg, mp = bctx.batch_autotune(scs, [sd.camera for sd in DESCS], [sd.params for sd in DESCS], sample_spp=1)
    assert mp > 0
    assert cfg["use_graph"] == 1 and cfg["bvh_width"] == 2
    assert bctx.batch_config()["paths_in_flight"] == cfg["paths_in_flight"]
    got, _ = _batch(bctx, scs, DESCS)
    bctx.set_batch_config()
    _same(got, _per_scene(bctx, scs, DESCS))


def test_batch_autotune_tries_both_widths(bctx, scs):
    """With the same scenes built with the 8-wide BVH (on the device) as the
    alternative, the autotuner picks a width; the batch renders with the
    chosen scenes give each instance its per-scene film."""
    c8 = g.Context(0, bvh_width=8)
    try:
        s8 = [g.Scene(sd, c8) for sd in DESCS]
        cams, prms = [sd.camera for sd in DESCS], [sd.params for sd in DESCS]
        cfg, mp = bctx.batch_autotune(scs, cams, prms, scenes_alt=s8, sample_spp=1)
        assert mp > 0 and cfg["bvh_width"] in (2, 8)
        chosen = s8 if cfg["bvh_width"] == 8 else scs
        got, _ = _batch(bctx, chosen, DESCS)
        bctx.set_batch_config()
        _same(got, _per_scene(bctx, chosen, DESCS))
        for sc in s8:
            sc.close()
    finally:
        c8.close()


def test_batch_more_instances_than_one_group(bctx):
    # more instances than the constant-memory table holds: consecutive groups
    descs = [scenes.cornell_box(res=8, spp=1 + k % 3, max_depth=3, spheres=bool(k % 2)) for k in range(150)]
    scs = [g.Scene(sd, bctx) for sd in descs]
    got, st = _batch(bctx, scs, descs)
    _same(got, _per_scene(bctx, scs, descs))
    assert st["paths"] == sum(sd.n_paths() for sd in descs)
