"""Film output fixtures (tests/golden/film_output.npz, made by the reference's
ImageIO compiled from its sources): the .png and .bmp writers store
ImageIO::toInt at gamma 2.2 of every channel, and the .hdr writer stores
Ward's RGBE (shared exponent from frexp of the largest component, mantissas
truncated). These pin the quantisation and the RGBE rule that the GPU film
output restates (gyt_film_quantize, gyt_film_save)."""
import numpy as np

from conftest import golden


def _rgbe(img):
    """RGBE bytes of a float image: m = max(r, g, b); below 1e-32 all zero;
    else frexp(m) = f * 2^e, channel = trunc(c * (f * 256 / m)), e + 128."""
    img = np.ascontiguousarray(img, np.float32)
    m = img.max(axis=2)
    f, e = np.frexp(m)
    with np.errstate(invalid="ignore", divide="ignore"):
        norm = (f.astype(np.float32) * np.float32(256.0)) / m
        ch = np.trunc(img * norm[..., None]).astype(np.int64)
    out = np.zeros(img.shape[:2] + (4,), np.uint8)
    ok = m >= np.float32(1e-32)
    out[..., :3] = np.where(ok[..., None], ch, 0).astype(np.uint8)
    out[..., 3] = np.where(ok, e + 128, 0).astype(np.uint8)
    return out


def test_png_and_bmp_store_the_same_bytes():
    g = golden("film_output.npz")
    assert np.array_equal(g["decoded_png"], g["decoded_bmp"])


def test_hdr_stores_ward_rgbe():
    # pixels with a negative component are left out: the reference's float to
    # byte conversion of a negative mantissa is undefined (no render produces one)
    g = golden("film_output.npz")
    ok = np.all(g["image"] >= 0, axis=2)
    assert ok.sum() > 500
    assert np.array_equal(_rgbe(g["image"])[ok], g["decoded_hdr"][ok])


def test_toint_range_and_monotone():
    g = golden("film_output.npz")
    x = g["x"]
    for k in ("toint_2.2", "toint_1.8", "toint_1"):
        v = g[k]
        assert v.min() == 0 and v.max() == 255
        order = np.argsort(x, kind="stable")
        assert np.all(np.diff(v[order]) >= 0)  # toInt is monotone in x
    # gamma 1 is plain rounding of the clamped value
    c = np.clip(x, 0, 1).astype(np.float32)
    assert np.array_equal(g["toint_1"], (c * np.float32(255) + np.float32(0.5)).astype(np.int32))
