"""Volumetric path tracing on the GPU (gyt_trace_volume_paths,
gyt_render_volume) against VolPathTracing of the reference compiled from its
sources (tests/golden/vpt_paths_*.npz, image_vpt_fog_64x64_8spp.npz), on the
Cornell box filled with a homogeneous medium. Needs a B200.

Per path the radiance must agree within relative 1e-4 of max(|L|, 1e-3) and
the path must use the same number of sampler dimensions. A path can branch
differently where a rounding decides (a scattering distance that lands on a
surface, a grazing shadow ray); those are counted and bounded."""
import dataclasses

import numpy as np
import pytest
import torch

from conftest import golden
import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu

def _halton_fog():
    sd = scenes.cornell_fog(res=48, spp=4, max_depth=6)
    return dataclasses.replace(sd, params=dataclasses.replace(sd.params, sampler="halton"))


# the fog ball: a closed material-less icosphere whose inside is the medium,
# entered and left through its faces (medium transitions both ways)
CASES = {"fog": lambda: scenes.cornell_fog(res=48, spp=4, max_depth=6),
         "fog_thick": lambda: scenes.cornell_fog(res=48, spp=4, max_depth=6, sigma_a=0.2, sigma_s=1.5, g=-0.4,
                                                 spheres=False),
         "fog_ball": lambda: scenes.fog_ball_box(res=48, spp=4, max_depth=6),
         "fog_halton": _halton_fog}


@pytest.mark.parametrize("name", list(CASES))
def test_volume_paths_match_reference(ctx, name):
    gd = golden("vpt_paths_%s.npz" % name)
    sc = g.Scene(CASES[name](), ctx)
    L, cur = sc.trace_volume_paths(gd["xys"])
    ref = gd["L"].astype(np.float64)
    rel = np.abs(L - ref).max(1) / np.maximum(np.abs(ref).max(1), 1e-3)
    same = cur == gd["cursor"]
    print(name, "paths within 1e-4: %.4f, same dims: %.4f, mean L %s vs %s" % (
        (rel < 1e-4).mean(), same.mean(), L.mean(0), ref.mean(0)))
    assert np.isfinite(L).all()
    assert same.mean() > 0.995
    assert (rel < 1e-4).mean() > 0.99


def test_volume_image_matches_reference(ctx):
    gd = golden("image_vpt_fog_64x64_8spp.npz")["film"].reshape(64, 64, 4).astype(np.float64)
    ref = gd[..., :3] / gd[..., 3:]
    sd = scenes.cornell_fog(res=64, spp=8, max_depth=6)
    sc = g.Scene(sd, ctx)
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.VolPathTracing(8, 6, equal_angular=False).Render(sc, cam)
    img = film.image.astype(np.float64)
    rel_mean = abs(img.mean() - ref.mean()) / ref.mean()
    rmse = np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    print("volume image: relative mean %.2e, relative RMSE %.4f" % (rel_mean, rmse))
    assert rel_mean < 5e-4 and rmse < 0.01


def test_volume_without_media_matches_path_tracing(ctx):
    """With no medium anywhere VolPathTracing draws the same sampler
    dimensions as PathTracing and reduces to it: on the Cornell box the two
    images agree."""
    sd = scenes.cornell_box(res=48, spp=8, max_depth=6)
    sc = g.Scene(sd, ctx)
    d_v = torch.zeros(48 * 48 * 4, dtype=torch.float64, device="cuda")
    ctx.render_volume_device(sc, sd.camera, sd.params, d_v.data_ptr())
    film = g.Film(48, 48)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.GpuPathTracing(8, 6).Render(sc, cam)
    pt = film.image.astype(np.float64)
    acc = d_v.view(48, 48, 4).cpu().numpy()
    v = acc[..., :3] / acc[..., 3:]
    rel = abs(v.mean() - pt.mean()) / pt.mean()
    print("VPT vs PT without media: relative mean %.2e" % rel)
    assert rel < 1e-4


def test_volume_device_accumulates(ctx):
    sd = scenes.cornell_fog(res=32, spp=2, max_depth=4)
    sc = g.Scene(sd, ctx)
    d = torch.zeros(32 * 32 * 4, dtype=torch.float64, device="cuda")
    st = ctx.render_volume_device(sc, sd.camera, sd.params, d.data_ptr())
    once = d.clone()
    ctx.render_volume_device(sc, sd.camera, sd.params, d.data_ptr())
    assert st["paths"] == 32 * 32 * 2 and once.sum() > 0
    assert torch.allclose(d, 2 * once, rtol=1e-9, atol=1e-12)


def test_volume_edge_sizes(ctx):
    sc = g.Scene(scenes.cornell_fog(res=16, spp=1, max_depth=3), ctx)
    L, cur = sc.trace_volume_paths(np.zeros((0, 3), np.uint32))
    assert L.shape == (0, 3) and cur.shape == (0,)
    L, cur = sc.trace_volume_paths(np.array([[0, 0, 0], [15, 15, 0]], np.uint32))
    assert L.shape == (2, 3) and np.isfinite(L).all() and np.all(cur >= 2)


def test_volume_rejects_bad_input(ctx):
    """Errors come back as status codes: an environment light is refused, a
    medium index out of range and a sample off the film are rejected."""
    sd = scenes.cornell_fog(res=16, spp=1, max_depth=3)
    d = torch.zeros(16 * 16 * 4, dtype=torch.float64, device="cuda")
    env = g.Scene(scenes.env_knot_small(), ctx)
    with pytest.raises(g.GytError):
        ctx.render_volume_device(env, sd.camera, sd.params, d.data_ptr())
    bad = dataclasses.replace(sd, tri_medium=np.where(sd.tri_medium >= 0, 1, -1).astype(np.int32))
    with pytest.raises(g.GytError):
        g.Scene(bad, ctx)
    sc = g.Scene(sd, ctx)
    with pytest.raises(g.GytError):
        sc.trace_volume_paths(np.array([[16, 0, 0]], np.uint32))
    # the context stays usable after the errors
    L, cur = sc.trace_volume_paths(np.array([[3, 4, 0]], np.uint32))
    assert np.isfinite(L).all() and cur[0] >= 2


# ---- equi-angular sampling (VolPathTracing's constructor default) ----------

def _equi(sd):
    return dataclasses.replace(sd, params=dataclasses.replace(sd.params, equi_angular=True))


EQ_CASES = {k: CASES[k] for k in ("fog", "fog_thick", "fog_ball")}


@pytest.mark.parametrize("name", list(EQ_CASES))
def test_equi_angular_paths_match_reference(ctx, name):
    """Per path against the reference's VolPathTracing with equalAngular =
    true (tests/golden/vpt_eq_paths_*.npz): the light and point drawn every
    bounce, the equi-angular distance in the medium, the connection to the
    light point."""
    gd = golden("vpt_eq_paths_%s.npz" % name)
    sd = _equi(EQ_CASES[name]())
    sc = g.Scene(sd, ctx)
    L, cur = sc.trace_volume_paths(gd["xys"])
    ref = gd["L"].astype(np.float64)
    rel = np.abs(L - ref).max(1) / np.maximum(np.abs(ref).max(1), 1e-3)
    same = cur == gd["cursor"]
    print(name, "equi-angular paths within 1e-4: %.4f, same dims: %.4f, mean L %s vs %s" % (
        (rel < 1e-4).mean(), same.mean(), L.mean(0), ref.mean(0)))
    assert np.isfinite(L).all()
    assert same.mean() > 0.995
    assert (rel < 1e-4).mean() > 0.99


def test_equi_angular_image_matches_reference(ctx):
    gd = golden("image_vpt_eq_fog_64x64_8spp.npz")["film"].reshape(64, 64, 4).astype(np.float64)
    ref = gd[..., :3] / gd[..., 3:]
    sd = scenes.cornell_fog(res=64, spp=8, max_depth=6)
    sc = g.Scene(sd, ctx)
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.VolPathTracing(8, 6).Render(sc, cam)  # equal_angular defaults to True, as the reference's constructor
    img = film.image.astype(np.float64)
    rel_mean = abs(img.mean() - ref.mean()) / ref.mean()
    rmse = np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    print("equi-angular volume image: relative mean %.2e, relative RMSE %.4f" % (rel_mean, rmse))
    assert rel_mean < 5e-4 and rmse < 0.01


def test_equi_angular_needs_an_area_light_and_is_volume_only(ctx):
    sd = _equi(scenes.cornell_fog(res=16, spp=1, max_depth=3))
    sc = g.Scene(sd, ctx)
    d = torch.zeros(16 * 16 * 4, dtype=torch.float64, device="cuda")
    # the path tracer does not take the volumetric flag
    with pytest.raises(g.GytError):
        ctx.render_device(sc, sd.camera, sd.params, d.data_ptr())
    dark = dataclasses.replace(sd, tri_emission=np.full_like(sd.tri_emission, -1))
    with pytest.raises(g.GytError):
        g.Scene(dark, ctx).trace_volume_paths(np.array([[3, 4, 0]], np.uint32))
    L, cur = sc.trace_volume_paths(np.array([[3, 4, 0]], np.uint32))
    assert np.isfinite(L).all() and cur[0] >= 2
