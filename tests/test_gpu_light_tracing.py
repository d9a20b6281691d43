"""Light tracing on the GPU (gyt_trace_light_paths, gyt_render_light_tracing)
against LightTracing of the reference compiled from its sources
(tests/golden/lt_paths_*.npz, image_lt_cornell_64x64_16spp.npz). Needs a B200.

Per photon, every vertex's camera join is compared: whether it lands on the
film, its pixel and its splatted RGB (FP32 on both sides, relative 1e-4 of
max(|L|, 1e-3)). Joins can differ where a rounding decides: a shadow ray that
grazes an edge or ends on the light, a raster position on a pixel boundary,
or a path that branches after such an event; they are counted and bounded."""
import numpy as np
import pytest
import torch

from conftest import golden
import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu

CASES = {"cornell_nospheres": lambda: scenes.cornell_box(res=64, spp=4, max_depth=6, spheres=False),
         "cornell": lambda: scenes.cornell_box(res=64, spp=4, max_depth=6),
         "mixed": lambda: scenes.mixed_materials_box(level=3, res=48, spp=4)}


@pytest.mark.parametrize("name", list(CASES))
def test_light_paths_match_reference(ctx, name):
    gd = golden("lt_paths_%s.npz" % name)
    sd = CASES[name]()
    got = g.Scene(sd, ctx).trace_light_paths(gd["photons"])
    ref = gd["records"]
    assert got.shape == ref.shape
    exists = (got[..., 0] >= 0) == (ref[..., 0] >= 0)
    same_on = got[..., 0] == ref[..., 0]
    both = (got[..., 0] == 1) & (ref[..., 0] == 1)
    same_px = np.all(got[..., 1:3] == ref[..., 1:3], axis=-1)
    # radiance compared on the joins both sides splat (the others carry no
    # splat; a missing vertex's GPU record is the sentinel (-1, 0, 0, 0, 0, 0))
    g3, r3 = got[both][:, 3:].astype(np.float64), ref[both][:, 3:].astype(np.float64)
    rel = np.zeros(both.shape)
    rel[both] = np.abs(g3 - r3).max(-1) / np.maximum(np.abs(r3).max(-1), 1e-3)
    ok = both & same_px & (rel < 1e-4)
    assert np.isfinite(g3).all()
    none = got[..., 0] < 0
    assert np.all(got[none][:, 1:] == 0)
    print(name, "same vertex count %.4f, same film flag %.4f, joins on film %d, matching %.4f" % (
        exists.mean(), same_on.mean(), both.sum(), ok.sum() / max(1, both.sum())))
    assert exists.mean() > 0.99
    assert same_on.mean() > 0.99
    assert ok.sum() > 0.98 * both.sum()


def test_light_tracing_image_matches_reference(ctx):
    ref = golden("image_lt_cornell_64x64_16spp.npz")["splat"].astype(np.float64)
    sd = scenes.cornell_box(res=64, spp=16, max_depth=6)
    sc = g.Scene(sd, ctx)
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.LightTracing(6, 16).Render(sc, cam)
    img = film.image.astype(np.float64)
    # the light itself (splats of its own vertices) dominates the mean; compare
    # the rest of the image too
    rel_mean = abs(img.mean() - ref.mean()) / ref.mean()
    lit = ref.max(axis=2) < 3.0
    rel_rest = abs(img[lit].mean() - ref[lit].mean()) / ref[lit].mean()
    rmse = np.sqrt(np.mean((img[lit] - ref[lit]) ** 2)) / np.sqrt(np.mean(ref[lit] ** 2))
    print("relative mean %.2e, away from the light %.2e, relative RMSE %.3f" % (rel_mean, rel_rest, rmse))
    assert rel_mean < 1e-3 and rel_rest < 5e-3 and rmse < 0.05


def test_light_tracing_device_accumulates_and_refuses_env(ctx):
    sd = scenes.cornell_box(res=32, spp=2, max_depth=4)
    sc = g.Scene(sd, ctx)
    d = torch.zeros(32 * 32 * 3, dtype=torch.float64, device="cuda")
    st = ctx.render_light_tracing_device(sc, sd.camera, sd.params, d.data_ptr())
    once = d.clone()
    ctx.render_light_tracing_device(sc, sd.camera, sd.params, d.data_ptr())
    assert st["paths"] == 32 * 32 * 2 and once.sum() > 0
    assert torch.allclose(d, 2 * once, rtol=1e-9, atol=1e-12)
    env = g.Scene(scenes.env_knot_small(), ctx)
    with pytest.raises(g.GytError):
        ctx.render_light_tracing_device(env, sd.camera, sd.params, d.data_ptr())
