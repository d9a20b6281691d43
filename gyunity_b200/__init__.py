"""gyunity_b200: the reference renderer's PathTracing integrator on B200.

Host-side mirror of the reference interfaces this component replaces
(xiaoyxue/Gyunity, paths inside Gyunity/src), over the C ABI in
include/gyt.h:

=========================  ==============================================
this module                reference
=========================  ==============================================
``Film``                   visual/Film.h (pixel buffer, SetImage)
``PinHoleCamera``          camera/PinholeCamera.h (GenerateRay set-up)
``Scene``                  visual/Scene.h + accelerator/BVHAccel.h
``GpuPathTracing.Render``  Integrator::Render (integrator/Integrator.h:20)
                           = TiledIntegrator::Render + PathTracing::Li
``Renderer.Render``        visual/Renderer.h:22-26
=========================  ==============================================

Errors raise ``GytError`` (the reference logs and exits, common/Core.h:160-166).
The CUDA library is required: there is no CPU fallback.
"""
import ctypes

import numpy as np

from . import scenes
from ._capi import GytError, load
from . import _capi as _c
from .scenes import Camera, RenderParams, SceneDesc

__all__ = ["Context", "Scene", "Film", "PinHoleCamera", "GpuPathTracing", "LightTracing", "VolPathTracing", "Renderer",
           "GytError",
           "SceneDesc", "Camera", "RenderParams", "scenes", "default_context"]


class Context:
    """A CUDA device with its stream and path pools (gyt_context)."""

    def __init__(self, device=0, capacity=None, bvh_width=None, bvh_builder=None):
        self._lib = load()
        h = ctypes.c_void_p()
        rc = self._lib.gyt_context_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise GytError(rc, "gyt_context_create(device=%d) failed" % device)
        self.handle = h
        self.device = device
        if capacity is not None:
            self.check(self._lib.gyt_context_set_capacity(self.handle, int(capacity)))
        if bvh_width is not None:
            self.check(self._lib.gyt_context_set_bvh_width(self.handle, int(bvh_width)))
        if bvh_builder is not None:
            code = {"host": _c.BVH_BUILD_HOST, "device": _c.BVH_BUILD_DEVICE}.get(bvh_builder, bvh_builder)
            self.check(self._lib.gyt_context_set_bvh_builder(self.handle, int(code)))

    def check(self, rc):
        if rc != 0:
            raise GytError(rc, self._lib.gyt_last_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self._lib.gyt_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_profile(self, mode):
        """0 off, 1 per-kernel event timing, 2 timing + traversal counters."""
        self.check(self._lib.gyt_context_set_profile(self.handle, int(mode)))

    def read_profile(self):
        p = _c.GytProfile()
        self.check(self._lib.gyt_profile_read(self.handle, ctypes.byref(p)))
        k, t = _c.KERNELS, _c.TRAVERSALS
        return {"ms": dict(zip(k, list(p.ms))), "launches": dict(zip(k, list(p.launches))),
                "rays": dict(zip(t, list(p.rays))), "node_visits": dict(zip(t, list(p.node_visits))),
                "tri_tests": dict(zip(t, list(p.tri_tests)))}

    def render_device(self, scene, camera, params, d_film_ptr):
        """gyt_render_device into a caller-owned device film (res_x*res_y*4 doubles)."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_render_device(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                               ctypes.c_void_p(d_film_ptr), ctypes.byref(st)))
        return {"paths": st.paths, "path_slots": st.path_slots, "iterations": st.iterations,
                "launches": st.launches, "ms": st.ms}

    def render_device_noalloc(self, scene, camera, params, d_film_ptr, paths_in_flight=_c.NOALLOC_MAX_PATHS):
        """gyt_render_device_noalloc: the same render with the paths in flight
        kept in the library's built-in scratch array, for callers that must
        not allocate GPU memory during the call. Returns the status code."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        return self._lib.gyt_render_device_noalloc(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                                   ctypes.c_void_p(d_film_ptr), int(paths_in_flight))

    # ---- differentiable rendering -----------------------------------------
    def diff_forward(self, scene, camera, params, d_film_ptr, d_path_L_ptr):
        """gyt_diff_forward: render into the device film and record every
        path's radiance (res_x*res_y*spp*3 floats at d_path_L_ptr)."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_diff_forward(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                              ctypes.c_void_p(d_film_ptr), ctypes.c_void_p(d_path_L_ptr),
                                              ctypes.byref(st)))
        return {"paths": st.paths, "iterations": st.iterations, "launches": st.launches, "ms": st.ms}

    def diff_backward(self, scene, camera, params, d_img_grad_ptr, d_film_ptr, d_path_L_ptr, d_grad_mat_ptr,
                      d_grad_em_ptr):
        """gyt_diff_backward: adds dLoss/dparams into the device gradient arrays."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_diff_backward(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                               ctypes.c_void_p(d_img_grad_ptr), ctypes.c_void_p(d_film_ptr),
                                               ctypes.c_void_p(d_path_L_ptr), ctypes.c_void_p(d_grad_mat_ptr),
                                               ctypes.c_void_p(d_grad_em_ptr), ctypes.byref(st)))
        return {"paths": st.paths, "iterations": st.iterations, "launches": st.launches, "ms": st.ms}

    def diff_backward_paths(self, scene, xys, delta, L_total, camera=None, params=None):
        """gyt_diff_backward_paths: gradient sums (n_materials, 4) and
        (n_emission, 3) of explicit paths with adjoint weights delta."""
        cam = _c.camera_struct(camera or scene.desc.camera)
        prm = _c.params_struct(params or scene.desc.params)
        xys = np.ascontiguousarray(xys, np.uint32).reshape(-1, 3)
        n = xys.shape[0]
        d = np.ascontiguousarray(delta, np.float32).reshape(n, 3)
        L = np.ascontiguousarray(L_total, np.float32).reshape(n, 3)
        nm, ne = scene.desc.mat_type.shape[0], scene.desc.emission.shape[0]
        gm = np.zeros((nm, 4), np.float64)
        ge = np.zeros((max(ne, 1), 3), np.float64)
        self.check(self._lib.gyt_diff_backward_paths(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                                     n, _c.ptr(xys), _c.ptr(d), _c.ptr(L), _c.ptr(gm), _c.ptr(ge)))
        return gm, ge[:ne]

    # ---- batched renders ---------------------------------------------------
    def set_batch_config(self, paths_in_flight=0, stride_blocks_per_sm=0, trace_blocks_per_sm=0, use_graph=True):
        c = _c.GytBatchConfig(int(paths_in_flight), int(stride_blocks_per_sm), int(trace_blocks_per_sm),
                              1 if use_graph else 0, 0)
        self.check(self._lib.gyt_context_set_batch_config(self.handle, ctypes.byref(c)))

    def batch_config(self):
        c = _c.GytBatchConfig()
        self.check(self._lib.gyt_context_get_batch_config(self.handle, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in _c.GytBatchConfig._fields_}

    @staticmethod
    def _batch_arrays(scenes, cameras, params):
        n = len(scenes)
        sc = (ctypes.c_void_p * n)(*[s.handle.value for s in scenes])
        cams = (_c.GytCamera * n)(*[_c.camera_struct(c) for c in cameras])
        prms = (_c.GytRenderParams * n)(*[_c.params_struct(p) for p in params])
        return n, sc, cams, prms

    def render_batch_device(self, scenes, cameras, params, d_film_ptrs):
        """gyt_render_batch_device: instance i = scenes[i] through cameras[i]
        with params[i], accumulated into the device film at d_film_ptrs[i]."""
        n, sc, cams, prms = self._batch_arrays(scenes, cameras, params)
        films = (ctypes.c_void_p * n)(*[int(p) for p in d_film_ptrs])
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_render_batch_device(self.handle, n, sc, cams, prms, films, ctypes.byref(st)))
        return {"paths": st.paths, "iterations": st.iterations, "launches": st.launches, "ms": st.ms}

    def render_batch(self, scenes, cameras, params, out=None):
        """gyt_render_batch: one host image (h, w, 3) per instance, written
        into ``out`` (C-contiguous float32 arrays of those shapes, e.g. kept
        from an earlier call or in pinned memory) when given."""
        n, sc, cams, prms = self._batch_arrays(scenes, cameras, params)
        if out is None:
            imgs = [np.empty((c.res_y, c.res_x, 3), np.float32) for c in cameras]
        else:
            imgs = list(out)
            if len(imgs) != n:
                raise ValueError("render_batch: %d output images for %d instances" % (len(imgs), n))
            for im, c in zip(imgs, cameras):
                if (not isinstance(im, np.ndarray) or im.dtype != np.float32 or im.shape != (c.res_y, c.res_x, 3)
                        or not im.flags.c_contiguous or not im.flags.writeable):
                    raise ValueError("render_batch: output images must be writeable C-contiguous float32 (h, w, 3)")
        outs = (ctypes.c_void_p * n)(*[im.ctypes.data for im in imgs])
        self.check(self._lib.gyt_render_batch(self.handle, n, sc, cams, prms, outs))
        return imgs

    def batch_autotune(self, scenes, cameras, params, scenes_alt=None, sample_spp=1):
        """gyt_batch_autotune: sets and returns the fastest batch
        configuration and its throughput (Mpaths/s) on a sample of the batch."""
        n, sc, cams, prms = self._batch_arrays(scenes, cameras, params)
        alt = None if scenes_alt is None else (ctypes.c_void_p * n)(*[s.handle.value for s in scenes_alt])
        best = _c.GytBatchConfig()
        mp = ctypes.c_float()
        self.check(self._lib.gyt_batch_autotune(self.handle, n, sc, alt, cams, prms, int(sample_spp),
                                                ctypes.byref(best), ctypes.byref(mp)))
        return {f: getattr(best, f) for f, _ in _c.GytBatchConfig._fields_}, mp.value

    # ---- parity / debug entry points --------------------------------------
    def bsdf_table(self, types, params, wo, u, we):
        """gyt_bsdf_table: the GPU's BxDF lobes for n cases (kind, 16
        parameters, wo, u, we): (n, 11) = sampled f, wi, pdf, then f and pdf
        toward we."""
        t = np.ascontiguousarray(types, np.uint32)
        n = t.shape[0]
        p = np.ascontiguousarray(params, np.float32).reshape(n, 16)
        v = np.ascontiguousarray(np.concatenate([np.reshape(wo, (n, 3)), np.reshape(u, (n, 3)),
                                                 np.reshape(we, (n, 3))], 1), np.float32)
        out = np.empty((n, 11), np.float32)
        self.check(self._lib.gyt_bsdf_table(self.handle, n, _c.ptr(t), _c.ptr(p), _c.ptr(v), _c.ptr(out)))
        return out

    def sobol(self, dims, indices):
        """sobol::sample (sampler/Sobol.h:46-61) for (dimension, index) pairs."""
        d = np.ascontiguousarray(dims, np.uint32)
        i = np.ascontiguousarray(indices, np.uint64)
        out = np.empty(d.shape[0], np.float32)
        self.check(self._lib.gyt_sobol(self.handle, d.shape[0], _c.ptr(d), _c.ptr(i), _c.ptr(out)))
        return out

    def render_volume_device(self, scene, camera, params, d_film_ptr):
        """gyt_render_volume_device: VolPathTracing into a device film
        (res_x*res_y*4 doubles, accumulated)."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_render_volume_device(self.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                                      ctypes.c_void_p(int(d_film_ptr)), ctypes.byref(st)))
        return {"paths": st.paths, "ms": st.ms}

    def render_light_tracing_device(self, scene, camera, params, d_splat_ptr):
        """gyt_render_light_tracing_device: LightTracing's splats accumulated
        into a device buffer of res_x*res_y*3 doubles."""
        cam = _c.camera_struct(camera)
        prm = _c.params_struct(params)
        st = _c.GytRenderStats()
        self.check(self._lib.gyt_render_light_tracing_device(self.handle, scene.handle, ctypes.byref(cam),
                                                             ctypes.byref(prm), ctypes.c_void_p(int(d_splat_ptr)),
                                                             ctypes.byref(st)))
        return {"paths": st.paths, "ms": st.ms}

    def film_quantize(self, d_film_ptr, res_x, res_y, gamma=2.2):
        """gyt_film_quantize: a device film (res_x*res_y*4 doubles) as 8-bit
        RGB (res_y, res_x, 3), ImageIO::toInt on the GPU."""
        out = np.empty((res_y, res_x, 3), np.uint8)
        self.check(self._lib.gyt_film_quantize(self.handle, ctypes.c_void_p(int(d_film_ptr)), res_x, res_y,
                                               float(gamma), _c.ptr(out)))
        return out

    def film_save(self, d_film_ptr, res_x, res_y, path):
        """gyt_film_save: Film::SaveImage of a device film (.png .bmp .hdr)."""
        self.check(self._lib.gyt_film_save(self.handle, ctypes.c_void_p(int(d_film_ptr)), res_x, res_y,
                                           str(path).encode()))

    def halton(self, dims, indices):
        """HaltonSampler with Faure permutations (sampler/Halton.h) for
        (dimension, index) pairs; dimensions >= 256 give 0."""
        d = np.ascontiguousarray(dims, np.uint32)
        i = np.ascontiguousarray(indices, np.uint64)
        out = np.empty(d.shape[0], np.float32)
        self.check(self._lib.gyt_halton(self.handle, d.shape[0], _c.ptr(d), _c.ptr(i), _c.ptr(out)))
        return out

    def halton_enum_index(self, res_x, res_y, s, x, y):
        """HaltonEnum::GetIndex (sampler/HaltonEnum.h) for (s, x, y)."""
        sxy = np.ascontiguousarray(np.stack([np.asarray(s), np.asarray(x), np.asarray(y)], 1), np.uint32)
        out = np.empty(sxy.shape[0], np.uint64)
        self.check(self._lib.gyt_halton_enum_index(self.handle, res_x, res_y, sxy.shape[0], _c.ptr(sxy),
                                                   _c.ptr(out)))
        return out

    def sobol_enum_index(self, res_x, res_y, s, x, y):
        """SobolEnum::GetIndex (sampler/SobolEnum.h:23-28) for (s, x, y)."""
        sxy = np.ascontiguousarray(np.stack([np.asarray(s), np.asarray(x), np.asarray(y)], 1), np.uint32)
        out = np.empty(sxy.shape[0], np.uint64)
        self.check(self._lib.gyt_sobol_enum_index(self.handle, res_x, res_y, sxy.shape[0], _c.ptr(sxy),
                                                  _c.ptr(out)))
        return out


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default


class Scene:
    """Scene + acceleration structure on the device (gyt_scene)."""

    def __init__(self, desc: SceneDesc, ctx: Context = None):
        self.ctx = ctx or default_context()
        self.desc = desc
        s, keep = _c.scene_struct(desc)
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx._lib.gyt_scene_create(self.ctx.handle, ctypes.byref(s), ctypes.byref(h)))
        self.handle = h

    def info(self):
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self.ctx._lib.gyt_scene_info(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"triangles": a.value, "bvh_nodes": b.value, "device_bytes": c.value}

    def set_materials(self, mat_params=None, emission=None, keep_light_sampling=False):
        """gyt_scene_set_materials: new material parameters (n_materials, 16)
        and/or emission rows (n_emission, 3); geometry and BVH are kept. With
        keep_light_sampling the light-selection distribution is not rebuilt."""
        mp = None if mat_params is None else np.ascontiguousarray(mat_params, np.float32)
        em = None if emission is None else np.ascontiguousarray(emission, np.float32)
        flags = _c.KEEP_LIGHT_SAMPLING if keep_light_sampling else 0
        self.ctx.check(self.ctx._lib.gyt_scene_set_materials(self.handle, _c.ptr(mp), _c.ptr(em), flags))

    def freeze_sampling(self, mat_params=None):
        """gyt_scene_freeze_sampling: BSDF sampling and pdfs from mat_params
        (n_materials, 16) while the GGX BSDF values follow the current
        parameters; None ends it. For difference checks of the adjoint."""
        mp = None if mat_params is None else np.ascontiguousarray(mat_params, np.float32)
        self.ctx.check(self.ctx._lib.gyt_scene_freeze_sampling(self.handle, _c.ptr(mp)))

    def read_bvh(self):
        """The binary BVH on the host: node slots (n, 16) float32 in the
        traversal layout and the scene triangle id of each leaf-order position."""
        n = ctypes.c_uint64()
        lib = self.ctx._lib
        self.ctx.check(lib.gyt_scene_read_bvh(self.handle, None, 0, None, 0, ctypes.byref(n)))
        nodes = np.zeros((n.value, 16), np.float32)
        ids = np.zeros(self.info()["triangles"], np.uint32)
        self.ctx.check(lib.gyt_scene_read_bvh(self.handle, _c.ptr(nodes), nodes.size, _c.ptr(ids), ids.size,
                                              ctypes.byref(n)))
        return nodes, ids

    def read_wide_bvh(self):
        """The 8-wide BVH on the host: nodes (n, 20) uint32 in the traversal
        layout and the scene triangle id of each leaf-order position."""
        n = ctypes.c_uint64()
        lib = self.ctx._lib
        self.ctx.check(lib.gyt_scene_read_wide_bvh(self.handle, None, 0, None, 0, ctypes.byref(n)))
        words = np.zeros((n.value, 20), np.uint32)
        ids = np.zeros(self.info()["triangles"], np.uint32)
        self.ctx.check(lib.gyt_scene_read_wide_bvh(self.handle, _c.ptr(words), words.size, _c.ptr(ids), ids.size,
                                                   ctypes.byref(n)))
        return words, ids

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.gyt_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def intersect(self, rays, any_hit=False):
        """BVHAccel::Intersect for rays (n, 7) = origin, direction, tmax.
        Returns prim ids (-1 miss; 1/0 for any_hit) and t, b1, b2."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 7)
        n = r.shape[0]
        prim = np.empty(n, np.int32)
        t, b1, b2 = (np.empty(n, np.float32) for _ in range(3))
        self.ctx.check(self.ctx._lib.gyt_intersect(self.ctx.handle, self.handle, n, _c.ptr(r), 1 if any_hit else 0,
                                                   _c.ptr(prim), _c.ptr(t), _c.ptr(b1), _c.ptr(b2)))
        return (prim.astype(bool),) if any_hit else (prim, t, b1, b2)

    def trace_volume_paths(self, xys, camera=None, params=None):
        """VolPathTracing::Li of explicit samples (n, 3) = x, y, s: radiance
        (n, 3) and the sampler dimensions each used."""
        cam = _c.camera_struct(camera or self.desc.camera)
        prm = _c.params_struct(params or self.desc.params)
        xys = np.ascontiguousarray(xys, np.uint32).reshape(-1, 3)
        n = xys.shape[0]
        L = np.empty((n, 3), np.float32)
        cur = np.empty(n, np.uint32)
        self.ctx.check(self.ctx._lib.gyt_trace_volume_paths(self.ctx.handle, self.handle, ctypes.byref(cam),
                                                            ctypes.byref(prm), n, _c.ptr(xys), _c.ptr(L),
                                                            _c.ptr(cur)))
        return L, cur

    def trace_light_paths(self, photons, camera=None, params=None):
        """LightTracing per photon index: (n, max_depth, 6) records of every
        vertex's camera join (on film 1/0 or -1, X, Y, splatted RGB)."""
        cam = _c.camera_struct(camera or self.desc.camera)
        p = params or self.desc.params
        prm = _c.params_struct(p)
        ids = np.ascontiguousarray(photons, np.uint64)
        out = np.empty((ids.shape[0], p.max_depth, 6), np.float32)
        self.ctx.check(self.ctx._lib.gyt_trace_light_paths(self.ctx.handle, self.handle, ctypes.byref(cam),
                                                           ctypes.byref(prm), ids.shape[0], _c.ptr(ids),
                                                           _c.ptr(out)))
        return out

    def trace_paths(self, xys, camera=None, params=None, decisions=False):
        """PathTracing::Li of explicit samples (n, 3) = x, y, s. Returns
        radiance (n, 3), Sobol' dimensions used and roulette-draw masks; with
        ``decisions`` also the shadow-occlusion and MIS-hit masks."""
        cam = _c.camera_struct(camera or self.desc.camera)
        prm = _c.params_struct(params or self.desc.params)
        xys = np.ascontiguousarray(xys, np.uint32).reshape(-1, 3)
        n = xys.shape[0]
        L = np.empty((n, 3), np.float32)
        cur = np.empty(n, np.uint32)
        rr, occ, mis = (np.empty(n, np.uint64) for _ in range(3))
        self.ctx.check(self.ctx._lib.gyt_trace_paths(self.ctx.handle, self.handle, ctypes.byref(cam),
                                                     ctypes.byref(prm), n, _c.ptr(xys), _c.ptr(L), _c.ptr(cur),
                                                     _c.ptr(rr), _c.ptr(occ), _c.ptr(mis)))
        return (L, cur, rr, occ, mis) if decisions else (L, cur, rr)


class VolPathTracing:
    """Drop-in for VolPathTracing(spp, maxDepth, sampler, samplerEnum,
    equalAngular = true) (integrator/VPT.h:12-19): volumetric path tracing
    through the scene's homogeneous media (SceneDesc.media, tri_medium);
    equal_angular selects equi-angular distance sampling about one light
    point per bounce, the reference constructor's default."""

    def __init__(self, spp, max_depth, sampler="sobol", equal_angular=True):
        if sampler not in _c.SAMPLERS:
            raise ValueError("sampler must be one of %s" % sorted(_c.SAMPLERS))
        self.params = RenderParams(int(spp), int(max_depth), 5, sampler, bool(equal_angular))

    def Render(self, scene, camera):
        ctx = scene.ctx
        cam = _c.camera_struct(camera.cam)
        prm = _c.params_struct(self.params)
        film = camera.GetFilm()
        rgb = np.empty((film.mResY, film.mResX, 3), np.float32)
        ctx.check(ctx._lib.gyt_render_volume(ctx.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                             _c.ptr(rgb)))
        film.SetImage(rgb)
        return film


class LightTracing:
    """Drop-in for LightTracing(sampler, maxDepth, spp) (integrator/LT.h:14-15):
    Render writes the splat image (Film::AddSplat) to the camera's film."""

    def __init__(self, max_depth, spp, sampler="sobol"):
        if sampler not in _c.SAMPLERS:
            raise ValueError("sampler must be one of %s" % sorted(_c.SAMPLERS))
        self.params = RenderParams(int(spp), int(max_depth), 5, sampler)

    def Render(self, scene, camera):
        ctx = scene.ctx
        cam = _c.camera_struct(camera.cam)
        prm = _c.params_struct(self.params)
        film = camera.GetFilm()
        rgb = np.empty((film.mResY, film.mResX, 3), np.float32)
        ctx.check(ctx._lib.gyt_render_light_tracing(ctx.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm),
                                                    _c.ptr(rgb)))
        film.SetImage(rgb)
        return film


class Film:
    """Film(w, h): the pixel buffer the integrator writes (visual/Film.h)."""

    def __init__(self, res_x, res_y):
        self.mResX, self.mResY = int(res_x), int(res_y)
        self.mAspectRatio = float(np.float32(res_x) / np.float32(res_y))
        self.image = np.zeros((self.mResY, self.mResX, 3), np.float32)

    def SetImage(self, image):
        """Film::SetImage (visual/Film.h:106-117): colour with weight 1."""
        self.image = np.asarray(image, np.float32).reshape(self.mResY, self.mResX, 3)

    def GetImage(self):
        return self.image

    def SaveImage(self, filename, ctx=None):
        """Film::SaveImage (visual/Film.cpp:6-9): the image (weight 1 per pixel,
        as Film::SetImage) through gyt_film_save; .png, .bmp or .hdr."""
        import torch
        ctx = ctx or default_context()
        film = np.ones((self.mResY, self.mResX, 4), np.float64)
        film[..., :3] = self.image
        d = torch.from_numpy(film.reshape(-1)).cuda()
        ctx.film_save(d.data_ptr(), self.mResX, self.mResY, filename)


class PinHoleCamera:
    """PinHoleCamera(film, position, lookAt, up, fovy, filmDistance)
    (camera/PinholeCamera.h:16-19)."""

    def __init__(self, film, position, look_at, up, fovy, film_distance):
        self.film = film
        self.cam = Camera(tuple(position), tuple(look_at), tuple(up), float(fovy), float(film_distance),
                          film.mResX, film.mResY)

    def GetFilm(self):
        return self.film

    def raster_to_world(self):
        out = np.empty(16, np.float64)
        c = _c.camera_struct(self.cam)
        rc = load().gyt_camera_raster_to_world(ctypes.byref(c), _c.ptr(out))
        if rc:
            raise GytError(rc, "raster_to_world")
        return out.reshape(4, 4)


class GpuPathTracing:
    """Drop-in for PathTracing(spp, maxDepth, sampler, samplerEnum)
    (integrator/PT.h:12). ``rr_depth``: roulette applies at bounce i > rr_depth
    (the reference hard-codes 5, integrator/PT.cpp:53). ``sampler``: "sobol"
    (SobolSampler + SobolEnum) or "halton" (HaltonSampler with Faure
    permutations + HaltonEnum)."""

    def __init__(self, spp, max_depth, rr_depth=5, ctx: Context = None, sampler="sobol"):
        if sampler not in _c.SAMPLERS:
            raise ValueError("sampler must be one of %s" % sorted(_c.SAMPLERS))
        self.params = RenderParams(int(spp), int(max_depth), int(rr_depth), sampler)
        self.ctx = ctx

    def Render(self, scene: Scene, camera: PinHoleCamera):
        ctx = scene.ctx
        cam = _c.camera_struct(camera.cam)
        prm = _c.params_struct(self.params)
        film = camera.GetFilm()
        rgb = np.empty((film.mResY, film.mResX, 3), np.float32)
        ctx.check(ctx._lib.gyt_render(ctx.handle, scene.handle, ctypes.byref(cam), ctypes.byref(prm), _c.ptr(rgb)))
        film.SetImage(rgb)
        return film


class Renderer:
    """Renderer(scene, camera, integrator, film).Render() (visual/Renderer.h:22-26)."""

    def __init__(self, scene, camera, integrator, film=None):
        self.scene, self.camera, self.integrator = scene, camera, integrator
        self.film = film or camera.GetFilm()

    def Render(self):
        return self.integrator.Render(self.scene, self.camera)
