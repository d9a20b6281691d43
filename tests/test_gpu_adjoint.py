"""Path replay adjoint on the GPU (gyt_diff_forward / gyt_diff_backward)
against the FP64 oracle adjoint, against itself through the image path, and
against central finite differences of the loss. Needs a B200."""
import numpy as np
import pytest
import torch

import gyunity_b200 as g
from gyunity_b200 import diff, scenes
from oracle.port import oracle as orc

pytestmark = pytest.mark.gpu


def _all_samples(sd):
    n = sd.camera.res_x * sd.camera.res_y * sd.params.spp
    k = np.arange(n, dtype=np.int64)
    pix, s = k // sd.params.spp, k % sd.params.spp
    return np.stack([pix % sd.camera.res_x, pix // sd.camera.res_x, s], 1).astype(np.uint32)


def _cases():
    p = scenes.inverse_params(groups=16, seed=7)
    a = scenes.inverse_box(p, level=3, res=32, spp=2, max_depth=5, rr_depth=5)
    b = scenes.inverse_box(p, level=3, res=32, spp=2, max_depth=6, rr_depth=1)
    c = scenes.mixed_materials_box(res=24, spp=2)
    return {"inverse_no_rr": a, "inverse_rr": b, "mixed": c}


CASES = _cases()


@pytest.mark.parametrize("name", list(CASES))
def test_path_adjoint_matches_fp64_oracle(ctx, name):
    sd = CASES[name]
    sc = g.Scene(sd, ctx)
    xys = _all_samples(sd)
    L, _, rr, occ, mis = sc.trace_paths(xys, decisions=True)
    # the paths whose forward radiance matches the FP64 replay (the per-path
    # parity criterion); the rest hit an exact tie between two triangles (rays
    # through the symmetric box's edges and corners), where either answer is
    # right and the paths continue differently
    Lo, _ = orc.OracleScene(sd).paths(xys[:, 0], xys[:, 1], xys[:, 2], precision=64, force_rr=rr, force_occ=occ,
                                      force_mis=mis)
    ok = np.abs(L - Lo).max(1) <= 1e-4 * np.maximum(np.abs(Lo).max(1), 1.0)
    print(name, "paths with matching radiance: %.4f" % ok.mean())
    assert ok.mean() > 0.98
    xys, L, rr, occ, mis = xys[ok], L[ok], rr[ok], occ[ok], mis[ok]
    delta = np.random.default_rng(11).normal(size=(xys.shape[0], 3)).astype(np.float32)
    gm, ge = ctx.diff_backward_paths(sc, xys, delta, L)
    om, oe, _ = orc.OracleScene(sd).adjoint(xys[:, 0], xys[:, 1], xys[:, 2], delta, precision=64, force_rr=rr,
                                            force_occ=occ, force_mis=mis)
    ref = np.concatenate([om.ravel(), oe.ravel()])
    got = np.concatenate([gm.ravel(), ge.ravel()])
    scale = np.abs(ref).max()
    assert scale > 0
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(name, "relative L2 error %.2e, worst entry %.2e of the largest" % (rel, np.abs(got - ref).max() / scale))
    assert rel < 1e-3
    assert np.abs(got - ref).max() <= 5e-3 * scale


def _spill_deltas(ctx, sd, xys, grad_img, film):
    """Per-path adjoint weights from an image gradient: the pixels each sample
    reaches (a sample on a pixel's left or lower edge also reaches the
    neighbour, as Film::AddSample's box filter), each divided by its weight."""
    cam = sd.camera
    m = int(np.ceil(np.log2(max(cam.res_x, cam.res_y))))
    res = np.float32(1 << m)
    idx = ctx.sobol_enum_index(cam.res_x, cam.res_y, xys[:, 2], xys[:, 0], xys[:, 1])
    su = ctx.sobol(np.zeros(len(idx), np.uint32), idx)
    sv = ctx.sobol(np.ones(len(idx), np.uint32), idx)
    x, y = xys[:, 0].astype(np.int64), xys[:, 1].astype(np.int64)
    u = res * su - x.astype(np.float32)
    v = res * sv - y.astype(np.float32)
    sx = (u == 0) & (x > 0)
    sy = (v == 0) & (y > 0)
    w = film[:, 3]
    gi = grad_img.reshape(-1, 3)
    d = np.zeros((xys.shape[0], 3), np.float64)
    for mx, my, on in ((0, 0, np.ones_like(sx)), (1, 0, sx), (0, 1, sy), (1, 1, sx & sy)):
        p = (y - my) * cam.res_x + (x - mx)
        p = np.where(on, p, 0)
        d += np.where(on[:, None], gi[p] / w[p][:, None], 0.0)
    return d.astype(np.float32), int(sx.sum() + sy.sum())


def test_image_adjoint_equals_path_adjoint(ctx):
    sd = CASES["inverse_no_rr"]
    r = diff.DiffRenderer(ctx, sd)
    p = scenes.inverse_params(groups=16, seed=7)
    img = r.forward(p)
    grad_img = torch.from_numpy(np.random.default_rng(3).normal(size=tuple(img.shape))).cuda()
    gimg = r.backward(grad_img)
    film = r.film.view(-1, 4).cpu().numpy()
    xys = _all_samples(sd)
    delta, spills = _spill_deltas(ctx, sd, xys, grad_img.cpu().numpy(), film)
    assert spills > 0  # the box-filter spill is exercised
    L = r.path_L.view(-1, 3).cpu().numpy()
    gm, ge = ctx.diff_backward_paths(r.scene, xys, delta, L)
    m = sd.param_materials
    np.testing.assert_allclose(gimg.albedo, gm[m, 0:3], rtol=1e-5, atol=1e-9 * np.abs(gm).max())
    np.testing.assert_allclose(gimg.alpha, gm[m, 3], rtol=1e-5, atol=1e-9 * np.abs(gm).max())
    np.testing.assert_allclose(gimg.radiance, ge, rtol=1e-5, atol=1e-9 * np.abs(ge).max())


def _fd_setup(ctx):
    hidden = scenes.inverse_params(groups=32, seed=7)
    sd = scenes.inverse_box(hidden, level=4, res=64, spp=8, max_depth=5, rr_depth=5)
    r = diff.DiffRenderer(ctx, sd)
    target = r.forward(hidden).clone()
    init = scenes.perturb_params(hidden, seed=8)
    return r, target, init


def _get(p, kind, i, c):
    if kind == "albedo":
        return p.albedo[i, c]
    if kind == "alpha":
        return p.alpha[i]
    return p.radiance[i, c]


def _with(p, kind, i, c, value):
    q = scenes.InverseParams(p.albedo.copy(), p.alpha.copy(), p.radiance.copy())
    if kind == "albedo":
        q.albedo[i, c] = value
    elif kind == "alpha":
        q.alpha[i] = value
    else:
        q.radiance[i, c] = value
    return q


def test_adjoint_matches_central_differences(ctx):
    r, target, init = _fd_setup(ctx)
    loss, grad = diff.loss_and_grad(r, init, target)
    assert loss > 0
    picks = [("albedo", i, c) for i, c in ((0, 0), (3, 1), (7, 2), (12, 0), (18, 1), (21, 2), (26, 0), (30, 1))]
    picks += [("alpha", i, 0) for i in (2, 9, 17, 28)] + [("radiance", i, c) for i, c in ((0, 0), (1, 1), (2, 2),
                                                                                            (3, 0))]
    h = 1e-3
    errs = {}
    for kind, i, c in picks:
        cur = _get(init, kind, i, c)
        # the scene stores float32: difference by the values actually rendered;
        # emitter steps keep the light-selection distribution, so that (like
        # the albedo) the estimator is exactly linear in the parameter; alpha
        # steps hold BSDF sampling and pdfs at the unstepped parameters
        # (gyt_scene_freeze_sampling), so that the difference quotient is the
        # detached-sampling derivative the adjoint computes
        keep = kind == "radiance"
        frozen = init if kind == "alpha" else None
        up, dn = np.float32(cur + h), np.float32(cur - h)
        fd = (diff.loss_at(r, _with(init, kind, i, c, up), target, keep, frozen) -
              diff.loss_at(r, _with(init, kind, i, c, dn), target, keep, frozen)) / (float(up) - float(dn))
        ad = _get(grad, kind, i, c)
        errs[(kind, i, c)] = (fd, ad, abs(fd - ad) / max(abs(fd), 1e-12))
    for k, v in errs.items():
        print(k, "fd %.6e adjoint %.6e rel %.2e" % v)
    for (kind, _, _), (fd, ad, rel) in errs.items():
        assert rel < (1e-2 if kind == "alpha" else 1e-3), (kind, fd, ad, rel)


def test_frozen_sampling_is_the_identity_at_the_frozen_parameters(ctx):
    """Sampling frozen at the current parameters renders the same film as
    free sampling (up to the refitted BSDF value's rounding), and the
    entry points that cannot honour it refuse a frozen scene."""
    r, target, init = _fd_setup(ctx)
    free = diff.loss_at(r, init, target)
    frozen = diff.loss_at(r, init, target, frozen_at=init)
    assert abs(frozen - free) <= 1e-5 * free
    r.freeze_sampling(init)
    try:
        with pytest.raises(g.GytError):
            r.backward(torch.zeros_like(target))
    finally:
        r.freeze_sampling(None)


def test_free_sampling_differences_converge_to_the_adjoint(ctx):
    """Differences with sampling free (the sampled directions move with alpha)
    are a different, much noisier estimator of the same derivative of the
    expected image. Over 64 disjoint sample sets of every pixel their mean
    agrees with the adjoint's within its standard error."""
    hidden = scenes.inverse_params(groups=32, seed=7)
    sd = scenes.inverse_box(hidden, level=4, res=64, spp=8, max_depth=5, rr_depth=5)
    sc = g.Scene(sd, ctx)
    p = scenes.perturb_params(hidden, seed=8)
    K, S = 64, sd.params.spp
    npix = sd.camera.res_x * sd.camera.res_y
    pix = np.repeat(np.arange(npix), S)
    base = np.stack([pix % sd.camera.res_x, pix // sd.camera.res_x, np.tile(np.arange(S), npix)], 1)
    xys = np.concatenate([base + np.array([0, 0, k * S]) for k in range(K)]).astype(np.uint32)
    # positive pixel weights (a loss gradient of one sign per pixel): the
    # functional's derivative is then not itself a cancellation of noise
    w = np.random.default_rng(5).uniform(0.5, 1.5, size=(npix, 3)).astype(np.float32)
    delta = np.tile(w[pix], (K, 1)) / np.float32(npix * S)

    def trace(q):
        mp, em = scenes.apply_inverse_params(sd, q)
        sc.set_materials(mp, em)
        return sc.trace_paths(xys)[0].reshape(K, -1, 3)

    L0 = trace(p)
    m = sd.param_materials
    adj = np.empty((K, len(m)))
    for k in range(K):
        sl = slice(k * npix * S, (k + 1) * npix * S)
        gm, _ = ctx.diff_backward_paths(sc, xys[sl], delta[sl], L0[k])
        adj[k] = gm[m, 3]
    d = delta.reshape(K, -1, 3).astype(np.float64)
    picks = np.argsort(-np.abs(adj.mean(0)))[:4]
    h = 1e-3
    for i in picks:
        up, dn = scenes.InverseParams(p.albedo, p.alpha.copy(), p.radiance), \
            scenes.InverseParams(p.albedo, p.alpha.copy(), p.radiance)
        up.alpha[i] = np.float32(p.alpha[i] + h)
        dn.alpha[i] = np.float32(p.alpha[i] - h)
        step = float(np.float32(up.alpha[i])) - float(np.float32(dn.alpha[i]))
        fd = ((d * (trace(up) - trace(dn))).sum((1, 2))) / step
        diffs = fd - adj[:, i]
        mean, se = diffs.mean(), diffs.std(ddof=1) / np.sqrt(K)
        print("alpha[%d] adjoint %.4e +- %.1e  free fd %.4e +- %.1e  (fd - adjoint) %.2e +- %.1e" %
              (i, adj[:, i].mean(), adj[:, i].std(ddof=1) / np.sqrt(K), fd.mean(), fd.std(ddof=1) / np.sqrt(K),
               mean, se))
        assert abs(mean) <= 4 * se + 1e-2 * abs(adj[:, i].mean())
    sc.close()


def test_inverse_rendering_reduces_the_loss(ctx):
    r, target, init = _fd_setup(ctx)
    p, hist = diff.optimize(r, target, init, iterations=20, lr=0.02)
    assert hist[-1] < 0.5 * hist[0]
    assert np.all(np.isfinite(p.flat()))
