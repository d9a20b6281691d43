"""The FP64 CPU adjoint of the oracle (path replay with detached sampling),
pinned by properties that need no GPU:

- d log f / d alpha of the GGX lobe against central differences of log f;
- albedo gradients against central differences of the FP64 path radiance
  (sampling does not depend on the albedo and roulette is off, so the
  weighted path radiance is a polynomial in the albedos and the two agree to
  rounding);
- emitter gradients by Euler's identity: every contribution holds exactly one
  emission factor, so sum(Le * dL/dLe) equals the weighted radiance itself;
- alpha gradients against central differences with the BSDF sampling held at
  the unperturbed alpha (the oracle's sampling-materials hook): that
  difference quotient is the detached-sampling derivative itself.
"""
import dataclasses

import numpy as np

from gyunity_b200 import scenes
from oracle.port import oracle as orc


def _unit(v):
    return v / np.linalg.norm(v)


def test_ggx_dlog_alpha_matches_finite_differences():
    rng = np.random.default_rng(3)
    for _ in range(300):
        a = rng.uniform(0.03, 0.9)
        wo = rng.normal(size=3)
        wi = rng.normal(size=3)
        wo[2], wi[2] = abs(wo[2]) + 0.02, abs(wi[2]) + 0.02
        wo, wi = _unit(wo), _unit(wi)
        h = 1e-6 * a
        fd = (orc.ggx_log_f(a + h, wo, wi) - orc.ggx_log_f(a - h, wo, wi)) / (2 * h)
        an = orc.ggx_dlog_alpha(a, wo, wi)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def _small():
    p = scenes.inverse_params(groups=8, seed=7)
    sd = scenes.inverse_box(p, level=2, res=8, spp=2, max_depth=4, rr_depth=4)
    n = sd.camera.res_x * sd.camera.res_y * sd.params.spp
    k = np.arange(n)
    pix, s = k // sd.params.spp, k % sd.params.spp
    x, y = pix % sd.camera.res_x, pix // sd.camera.res_x
    delta = np.random.default_rng(5).normal(size=(n, 3)).astype(np.float32)
    return sd, (x, y, s), delta


def _weighted(sd, xys, delta, occ=None, mis=None, sampling=None):
    o_ = orc.OracleScene(sd)
    if sampling is not None:
        o_.set_sampling_materials(sampling)
    L, _, _, o, m = o_.paths(*xys, precision=64, force_occ=occ, force_mis=mis, return_decisions=True)
    return float((L * delta.astype(np.float64)).sum()), o, m


def test_albedo_gradient_matches_finite_differences():
    sd, xys, delta = _small()
    base, occ, mis = _weighted(sd, xys, delta)
    gm, ge, L = orc.OracleScene(sd).adjoint(*xys, delta, precision=64, force_occ=occ, force_mis=mis)
    assert abs(float((L * delta).sum()) - base) <= 1e-9 * abs(base)
    for m in sd.param_materials[:4]:
        for c in range(3):
            # the parameters are float32: difference by the steps actually stored
            mp_up, mp_dn = sd.mat_params.copy(), sd.mat_params.copy()
            mp_up[m, c] += np.float32(1e-4)
            mp_dn[m, c] -= np.float32(1e-4)
            up, _, _ = _weighted(dataclasses.replace(sd, mat_params=mp_up), xys, delta, occ, mis)
            dn, _, _ = _weighted(dataclasses.replace(sd, mat_params=mp_dn), xys, delta, occ, mis)
            fd = (up - dn) / (float(mp_up[m, c]) - float(mp_dn[m, c]))
            assert abs(fd - gm[m, c]) <= 1e-6 * max(1.0, abs(fd)), (m, c, fd, gm[m, c])


def test_emitter_gradient_euler_identity():
    sd, xys, delta = _small()
    base, occ, mis = _weighted(sd, xys, delta)
    gm, ge, _ = orc.OracleScene(sd).adjoint(*xys, delta, precision=64, force_occ=occ, force_mis=mis)
    assert abs(float((sd.emission.astype(np.float64) * ge).sum()) - base) <= 1e-9 * abs(base)


def test_alpha_gradient_matches_frozen_sampling_differences():
    sd, xys, delta = _small()
    base, occ, mis = _weighted(sd, xys, delta)
    gm, _, _ = orc.OracleScene(sd).adjoint(*xys, delta, precision=64, force_occ=occ, force_mis=mis)
    checked = 0
    for m in sd.param_materials:
        mp_up, mp_dn = sd.mat_params.copy(), sd.mat_params.copy()
        for mp, sgn in ((mp_up, 1), (mp_dn, -1)):
            mp[m, 6] += np.float32(sgn * 1e-4)
            mp[m, 7] = mp[m, 6]
        up, _, _ = _weighted(dataclasses.replace(sd, mat_params=mp_up), xys, delta, occ, mis, sd.mat_params)
        dn, _, _ = _weighted(dataclasses.replace(sd, mat_params=mp_dn), xys, delta, occ, mis, sd.mat_params)
        fd = (up - dn) / (float(mp_up[m, 6]) - float(mp_dn[m, 6]))
        assert abs(fd - gm[m, 3]) <= 1e-5 * max(1.0, abs(fd)), (m, fd, gm[m, 3])
        checked += abs(fd) > 1e-6
    assert checked >= 4
