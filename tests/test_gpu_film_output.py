"""Film output on the GPU (gyt_film_quantize, gyt_film_save) against the
reference's ImageIO (tests/golden/film_output.npz). Needs a B200.

Tolerance: the quantisation is ImageIO::toInt in float; the GPU's powf and
the host C library's may differ in the last bit, which moves a value across
a rounding boundary of * 255 + 0.5 for about one channel in 10^5: at most one
channel in 10^4 may differ, and by one step only. RGBE bytes are exact."""
import os

import numpy as np
import pytest
import torch

from conftest import golden
from image_tools import read_hdr_rgbe, read_rgb8
import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu


def _film(img):
    h, w = img.shape[:2]
    f = np.ones((h, w, 4), np.float64)
    f[..., :3] = img
    return torch.from_numpy(f.reshape(-1)).cuda(), w, h


def _close(a, b):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    return d.max() <= 1 and (d > 0).mean() <= 1e-4


@pytest.mark.parametrize("gamma", [2.2, 1.8, 1.0])
def test_quantize_matches_toint(ctx, gamma):
    gd = golden("film_output.npz")
    x = gd["x"]
    n = x.shape[0]
    w = 101
    h = (n + w - 1) // w
    img = np.zeros((h * w, 3), np.float32)
    img[:n] = x[:, None]
    f, w_, h_ = _film(img.reshape(h, w, 3))
    q = ctx.film_quantize(f.data_ptr(), w_, h_, gamma).reshape(-1, 3)[:n]
    ref = gd["toint_%g" % gamma]
    for c in range(3):
        assert _close(q[:, c], ref), (gamma, int((q[:, c] != ref).sum()))


@pytest.mark.parametrize("ext", ["png", "bmp", "hdr"])
def test_save_matches_reference_writer(ctx, tmp_path, ext):
    gd = golden("film_output.npz")
    img = gd["image"]
    f, w, h = _film(img)
    path = str(tmp_path / ("film." + ext))
    ctx.film_save(f.data_ptr(), w, h, path)
    if ext == "hdr":
        ok = np.all(img >= 0, axis=2)  # negative components: undefined in the reference's writer
        assert np.array_equal(read_hdr_rgbe(path)[ok], gd["decoded_hdr"][ok])
    else:
        assert _close(read_rgb8(path), gd["decoded_" + ext])


def test_rendered_film_saves_its_quantized_bytes(ctx, tmp_path):
    sd = scenes.cornell_box(res=64, spp=4)
    sc = g.Scene(sd, ctx)
    f = torch.zeros(64 * 64 * 4, dtype=torch.float64, device="cuda")
    ctx.render_device(sc, sd.camera, sd.params, f.data_ptr())
    q = ctx.film_quantize(f.data_ptr(), 64, 64)
    for ext in ("png", "bmp"):
        path = str(tmp_path / ("r." + ext))
        ctx.film_save(f.data_ptr(), 64, 64, path)
        assert np.array_equal(read_rgb8(path), q)
    # the Python Film (weight 1 per pixel, Film::SetImage) through the same path
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.GpuPathTracing(4, sd.params.max_depth, sd.params.rr_depth).Render(sc, cam)
    path = str(tmp_path / "py.png")
    film.SaveImage(path, ctx)
    c = np.clip(film.image, 0, 1).astype(np.float32)
    host = (np.power(c, np.float32(1) / np.float32(2.2)) * np.float32(255) + np.float32(0.5)).astype(np.int32)
    assert _close(read_rgb8(path), host.astype(np.uint8))


def test_bad_requests_are_rejected(ctx, tmp_path):
    f = torch.ones(4 * 4 * 4, dtype=torch.float64, device="cuda")
    with pytest.raises(g.GytError):
        ctx.film_save(f.data_ptr(), 4, 4, str(tmp_path / "x.jpg"))
    with pytest.raises(g.GytError):
        ctx.film_quantize(f.data_ptr(), 0, 4)
    with pytest.raises(g.GytError):
        ctx.film_save(f.data_ptr(), 4, 4, str(tmp_path / "no_such_dir" / "x.png"))
    assert not os.path.exists(tmp_path / "x.jpg")
