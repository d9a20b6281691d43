"""The Halton sampler on the GPU (HaltonSampler with Faure permutations +
HaltonEnum, selected by GYT_SAMPLER_HALTON) against the reference's golden
vectors and the FP64 oracle. Needs a B200."""
import numpy as np
import pytest
import torch

from conftest import golden
import gyunity_b200 as g
from gyunity_b200 import scenes
from oracle.port import oracle as orc
from test_gpu_parity import _replay

pytestmark = pytest.mark.gpu


def _halton(sd):
    sd.params.sampler = "halton"
    return sd


def test_halton_bit_exact(ctx):
    gd = golden("halton.npz")
    got = ctx.halton(gd["dims"], gd["indices"])
    assert np.array_equal(got.view(np.uint32), gd["values"].view(np.uint32))


@pytest.mark.parametrize("res", ["256x256", "1024x1024", "1920x1080", "100x60", "1x1", "7x1", "1x5"])
def test_halton_enumeration_bit_exact(ctx, res):
    gd = golden("henum.npz")
    rx, ry = map(int, res.split("x"))
    sxy = gd[res + "_sxy"]
    assert np.array_equal(ctx.halton_enum_index(rx, ry, sxy[:, 0], sxy[:, 1], sxy[:, 2]), gd[res + "_index"])


def test_halton_edge_cases(ctx):
    # index 0, both sides of 2^32 (the 32- and 64-bit digit loops), the top of
    # the 64-bit range, the last dimension and dimensions past it
    dims = np.array([0, 1, 2, 255, 256, 1000, 1, 3, 254, 0, 7], np.uint32)
    idx = np.array([0, 0, (1 << 32) - 1, 1 << 32, 5, 5, (1 << 64) - 1, (1 << 63) + 17, (1 << 40) + 3,
                    (1 << 64) - 1, 3486784400], np.uint64)
    assert np.array_equal(ctx.halton(dims, idx).view(np.uint32), orc.halton(dims, idx).view(np.uint32))
    assert ctx.halton(np.zeros(0, np.uint32), np.zeros(0, np.uint64)).shape == (0,)


@pytest.mark.parametrize("name", ["cornell_nospheres", "mixed"])
def test_halton_per_path_radiance_matches_fp64_replay(ctx, name):
    sd = _halton({"cornell_nospheres": scenes.cornell_box(spheres=False),
                  "mixed": scenes.mixed_materials_box(level=3, res=64)}[name])
    xys = golden("paths_%s_halton.npz" % name)["xys"]
    rel, same_cursor, flips, _ = _replay(sd, xys, ctx)
    ok = rel < 1e-4  # FP32 path vs FP64 replay of the same path, relative to max(|L|, 1e-3)
    print(name, "paths within 1e-4:", ok.mean(), "same dims:", same_cursor.mean(), "decision flips:", flips)
    assert same_cursor.mean() > 0.995
    assert ok.mean() > 0.99
    assert flips < 0.05


def test_halton_per_path_radiance_matches_reference(ctx):
    gd = golden("paths_cornell_nospheres_halton.npz")
    sc = g.Scene(_halton(scenes.cornell_box(spheres=False)), ctx)
    L, cur, _ = sc.trace_paths(gd["xys"])
    ref = gd["L"].astype(np.float64)
    rel = np.abs(L - ref).max(1) / np.maximum(np.abs(ref).max(1), 1e-3)
    assert (cur == gd["cursor"]).mean() > 0.995
    assert (rel < 1e-4).mean() > 0.95


def test_halton_render_matches_reference_image(ctx):
    gd = golden("image_cornell_64x64_4spp_halton.npz")["film"].reshape(64, 64, 4).astype(np.float64)
    sd = scenes.cornell_box(res=64, spp=4)
    sc = g.Scene(sd, ctx)
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.GpuPathTracing(4, sd.params.max_depth, sd.params.rr_depth, sampler="halton").Render(sc, cam)
    ref = gd[..., :3] / gd[..., 3:]
    img = film.image.astype(np.float64)
    # a few paths branch differently after a glass bounce; one of them is a
    # bright caustic in the reference image (see the oracle's image test)
    close = (np.abs(img - ref).max(2) <= 1e-3).mean()
    print("pixels within 1e-3:", close, "mean", img.mean(), ref.mean())
    assert close > 0.9
    assert abs(img.mean() - ref.mean()) < 1e-2 * ref.mean()


def test_halton_and_sobol_instances_in_one_batch(ctx):
    # the sampler is per instance: a batch mixing both gives each instance the
    # film of its own per-scene render
    descs = [scenes.cornell_box(res=64, spp=4), _halton(scenes.cornell_box(res=64, spp=4)),
             _halton(scenes.mixed_materials_box(level=3, res=48, spp=3))]
    scs = [g.Scene(sd, ctx) for sd in descs]
    cams = [sd.camera for sd in descs]
    prms = [sd.params for sd in descs]
    ref = []
    for sc, sd in zip(scs, descs):
        f = torch.zeros(sd.camera.res_x * sd.camera.res_y * 4, dtype=torch.float64, device="cuda")
        ctx.render_device(sc, sd.camera, sd.params, f.data_ptr())
        ref.append(f)
    films = [torch.zeros_like(f) for f in ref]
    ctx.render_batch_device(scs, cams, prms, [f.data_ptr() for f in films])
    torch.cuda.synchronize()
    for a, b in zip(films, ref):
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-12)
    assert not torch.allclose(ref[0], ref[1])  # the two samplers give different images of one scene
