"""Differentiable rendering on top of the C ABI's path replay adjoint
(gyt_diff_forward / gyt_diff_backward): a forward/backward pair shaped like a
torch.autograd.Function, the L2 image loss and the inverse-rendering loop
(Adam) over per-group albedo, GGX alpha and emitter radiance.

The renders and gradients run in the native library; torch holds the device
buffers (film, per-path radiance, image, gradients) and runs the optimiser.
"""
import numpy as np
import torch

from . import Scene, scenes


class DiffRenderer:
    """One scene, camera and sample count, rendered and differentiated with
    respect to the InverseParams of an inverse_box scene (materials listed in
    desc.param_materials, emission rows in order)."""

    def __init__(self, ctx, desc, scene: Scene = None):
        self.ctx = ctx
        self.desc = desc
        self.scene = scene or Scene(desc, ctx)
        cam, prm = desc.camera, desc.params
        self.npix = cam.res_x * cam.res_y
        dev = "cuda:%d" % ctx.device
        self.film = torch.zeros(self.npix * 4, dtype=torch.float64, device=dev)
        self.path_L = torch.zeros(self.npix * prm.spp * 3, dtype=torch.float32, device=dev)
        self.nm, self.ne = desc.mat_type.shape[0], desc.emission.shape[0]
        self.grad_mat = torch.zeros(self.nm * 4, dtype=torch.float64, device=dev)
        self.grad_em = torch.zeros(max(self.ne, 1) * 3, dtype=torch.float64, device=dev)
        self.last = {}

    def set_params(self, p: "scenes.InverseParams", keep_light_sampling=False):
        mp, em = scenes.apply_inverse_params(self.desc, p)
        self.scene.set_materials(mp, em, keep_light_sampling=keep_light_sampling)

    def freeze_sampling(self, p: "scenes.InverseParams" = None):
        """Holds BSDF sampling and pdfs at the parameters p for the following
        forwards (gyt_scene_freeze_sampling); None ends it. Forwards at
        parameters stepped about p then differ exactly by the detached-sampling
        derivative the adjoint computes."""
        if p is None:
            self.scene.freeze_sampling(None)
            return
        mp, _ = scenes.apply_inverse_params(self.desc, p)
        self.scene.freeze_sampling(mp)

    def forward(self, p: "scenes.InverseParams", keep_light_sampling=False):
        """Renders with parameters p; returns the image (h, w, 3) on the
        device in float64 (colour / weight per pixel of the FP64 film, the
        values gyt_render rounds to float). keep_light_sampling keeps the
        light-selection distribution of the previous emission."""
        self.set_params(p, keep_light_sampling)
        self.film.zero_()
        st = self.ctx.diff_forward(self.scene, self.desc.camera, self.desc.params, self.film.data_ptr(),
                                   self.path_L.data_ptr())
        self.last["forward_ms"] = st["ms"]
        f = self.film.view(-1, 4)
        cam = self.desc.camera
        return (f[:, :3] / f[:, 3:4]).view(cam.res_y, cam.res_x, 3)

    def backward(self, grad_image):
        """dLoss/dparams for dLoss/dImage (h, w, 3) of the last forward:
        returns InverseParams-shaped float64 numpy gradients."""
        g = grad_image.to(torch.float32).contiguous()
        self.grad_mat.zero_()
        self.grad_em.zero_()
        st = self.ctx.diff_backward(self.scene, self.desc.camera, self.desc.params, g.data_ptr(),
                                    self.film.data_ptr(), self.path_L.data_ptr(), self.grad_mat.data_ptr(),
                                    self.grad_em.data_ptr())
        self.last["backward_ms"] = st["ms"]
        gm = self.grad_mat.view(self.nm, 4).cpu().numpy()
        ge = self.grad_em.view(-1, 3)[:self.ne].cpu().numpy()
        m = self.desc.param_materials
        return scenes.InverseParams(gm[m, 0:3].copy(), gm[m, 3].copy(), ge.copy())


class PathReplayRender(torch.autograd.Function):
    """image = render(albedo (g, 3), alpha (g,), radiance (e, 3)); backward by
    path replay. Parameters are float64 tensors (any device)."""

    @staticmethod
    def forward(ctx, albedo, alpha, radiance, renderer: DiffRenderer):
        p = scenes.InverseParams(albedo.detach().cpu().numpy(), alpha.detach().cpu().numpy(),
                                 radiance.detach().cpu().numpy())
        ctx.renderer = renderer
        ctx.devs = (albedo.device, alpha.device, radiance.device)
        return renderer.forward(p)

    @staticmethod
    def backward(ctx, grad_image):
        g = ctx.renderer.backward(grad_image)
        da, dl, dr = ctx.devs
        return (torch.from_numpy(g.albedo).to(da), torch.from_numpy(g.alpha).to(dl),
                torch.from_numpy(g.radiance).to(dr), None)


def l2_loss(image, target):
    """Mean squared error over pixels and channels."""
    return ((image - target) ** 2).mean()


def loss_and_grad(renderer: DiffRenderer, p: "scenes.InverseParams", target):
    """Loss at p and its gradient (InverseParams of float64) by one forward
    and one adjoint pass."""
    img = renderer.forward(p)
    diff = img - target
    loss = float((diff.double() ** 2).mean().item())
    grad_img = 2.0 * diff / diff.numel()
    return loss, renderer.backward(grad_img)


def loss_at(renderer: DiffRenderer, p: "scenes.InverseParams", target, keep_light_sampling=False,
            frozen_at: "scenes.InverseParams" = None):
    """The loss of a forward at p; with frozen_at, BSDF sampling and pdfs are
    held at those parameters during the forward."""
    if frozen_at is not None:
        renderer.freeze_sampling(frozen_at)
    try:
        img = renderer.forward(p, keep_light_sampling)
    finally:
        if frozen_at is not None:
            renderer.freeze_sampling(None)
    return float(((img - target).double() ** 2).mean().item())


def clamp_params(p: "scenes.InverseParams"):
    return scenes.InverseParams(np.clip(p.albedo, 0.01, 1.0), np.clip(p.alpha, 0.02, 1.0),
                                np.clip(p.radiance, 0.01, None))


def optimize(renderer: DiffRenderer, target, init: "scenes.InverseParams", iterations=200, lr=0.02, log=None):
    """Adam (torch.optim.Adam, lr) on albedo, alpha and radiance through
    PathReplayRender, parameters clamped to their valid ranges after every
    step. Returns the final parameters and the loss history."""
    dev = target.device
    a = torch.tensor(init.albedo, dtype=torch.float64, device=dev, requires_grad=True)
    al = torch.tensor(init.alpha, dtype=torch.float64, device=dev, requires_grad=True)
    r = torch.tensor(init.radiance, dtype=torch.float64, device=dev, requires_grad=True)
    opt = torch.optim.Adam([a, al, r], lr=lr)
    hist = []
    for it in range(iterations):
        opt.zero_grad()
        img = PathReplayRender.apply(a, al, r, renderer)
        loss = l2_loss(img.double(), target.double())
        loss.backward()
        opt.step()
        with torch.no_grad():
            a.clamp_(0.01, 1.0)
            al.clamp_(0.02, 1.0)
            r.clamp_(min=0.01)
        hist.append(float(loss.item()))
        if log:
            log(it, hist[-1])
    p = scenes.InverseParams(a.detach().cpu().numpy(), al.detach().cpu().numpy(), r.detach().cpu().numpy())
    return p, hist
