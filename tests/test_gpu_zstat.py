"""Per-pixel z-test of the GPU's converged image against the reference's
(PathTracing of the reference compiled from its sources; per-pixel mean and
variance over samples 0..spp-1 in tests/golden/zstat_*.npz), with the RMSE
stated. Needs a B200.

Two comparisons per scene, both at the reference's spp:
- independent: the GPU's samples spp..2 spp-1 of every pixel (a disjoint set
  of the same Sobol' sequence) against the reference's 0..spp-1; Welch's
  z = (m_gpu - m_ref) / sqrt(v_gpu / spp + v_ref / spp) per pixel and
  channel. The reference against itself on the same two sets gives 0.08% of
  Cornell-box pixels beyond |z| = 3 (disjoint Sobol' sets are less noisy
  than independent random ones), so a fraction above 0.5%, or a mean z
  away from 0, means the two estimators differ;
- same samples: the GPU's samples 0..spp-1 against the reference's, the
  same paths up to rounding-decided events.
Pixels whose variance is 0 on both sides must have equal means."""
import dataclasses

import numpy as np
import pytest

from conftest import golden
import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = {
    "cornell_256x256_16spp": lambda: scenes.cornell_box(res=256, spp=16),
    "env_knot_96x54_16spp": lambda: dataclasses.replace(
        scenes.env_knot_small(), params=dataclasses.replace(scenes.env_knot_small().params, spp=16)),
    "inverse_128x128_16spp": lambda: scenes.inverse_box(level=5, res=128, spp=16, max_depth=8, rr_depth=8),
}


def _moments(sc, W, H, s0, S):
    pix = np.repeat(np.arange(W * H), S)
    xys = np.stack([pix % W, pix // W, np.tile(np.arange(s0, s0 + S), W * H)], 1).astype(np.uint32)
    L = sc.trace_paths(xys)[0].astype(np.float64).reshape(W * H, S, 3)
    return L.mean(1), L.var(1, ddof=1)


def _z(ma, va, mb, vb, S):
    se = np.sqrt(va / S + vb / S)
    ok = se > 0
    z = np.where(ok, (ma - mb) / np.where(ok, se, 1.0), 0.0)
    return z, ok


@pytest.mark.parametrize("name", list(SCENES))
def test_per_pixel_z(ctx, name):
    gd = golden("zstat_%s.npz" % name)
    sd = SCENES[name]()
    W, H = int(gd["res"][0]), int(gd["res"][1])
    S = int(gd["spp"])
    assert (sd.camera.res_x, sd.camera.res_y, sd.params.spp) == (W, H, S)
    mr, vr = gd["mean"].astype(np.float64), gd["var"].astype(np.float64)
    sc = g.Scene(sd, ctx)
    mi, vi = _moments(sc, W, H, S, S)   # disjoint samples
    ms, vs = _moments(sc, W, H, 0, S)   # the reference's samples
    sc.close()
    zi, oki = _z(mi, vi, mr, vr, S)
    zs, oks = _z(ms, vs, mr, vr, S)
    rms = np.sqrt(np.mean(mr ** 2))
    rmse_i = np.sqrt(np.mean((mi - mr) ** 2))
    rmse_s = np.sqrt(np.mean((ms - mr) ** 2))
    fi, fs = float((np.abs(zi) > 3).mean()), float((np.abs(zs) > 3).mean())
    print("%s: independent samples |z|>3 %.4f%% (mean z %+.4f), RMSE %.3e (%.2f%% of RMS); same samples |z|>3 "
          "%.4f%%, RMSE %.3e; zero-variance pixels %.2f%%" % (name, 100 * fi, zi[oki].mean(), rmse_i,
                                                              100 * rmse_i / rms, 100 * fs, rmse_s,
                                                              100 * (~oki).mean()))
    assert fi < 0.005
    assert abs(zi[oki].mean()) < 0.02
    assert fs < 0.005
    # a pixel without variance on both sides (a constant radiance: the
    # background, an emitter seen directly) must agree
    assert np.all(np.abs(mi - mr)[~oki] <= 1e-5 * np.maximum(np.abs(mr[~oki]), 1e-3))
