"""ctypes binding of the native C ABI (include/gyt.h) in libgyunity_b200.so.

There is no fallback: if the library is missing or was built for another
ABI, loading raises ``GytError`` with the reason.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgyunity_b200.so")

GYT_OK = 0
STATUS = {0: "GYT_OK", 1: "GYT_ERR_INVALID", 2: "GYT_ERR_CUDA", 3: "GYT_ERR_OUT_OF_MEMORY",
          4: "GYT_ERR_UNSUPPORTED", 5: "GYT_ERR_WATCHDOG"}

# Every entry point include/gyt.h declares (checked by the CPU tests).
EXPORTS = ["gyt_context_create", "gyt_context_destroy", "gyt_last_error", "gyt_context_set_capacity",
           "gyt_context_set_profile", "gyt_profile_read", "gyt_context_set_bvh_width",
           "gyt_context_set_bvh_builder", "gyt_scene_create", "gyt_scene_destroy", "gyt_scene_info",
           "gyt_scene_read_bvh", "gyt_render", "gyt_render_device",
           "gyt_trace_paths", "gyt_intersect", "gyt_sobol", "gyt_sobol_enum_index", "gyt_halton",
           "gyt_halton_enum_index", "gyt_camera_raster_to_world", "gyt_film_quantize", "gyt_film_save",
           "gyt_render_light_tracing", "gyt_render_light_tracing_device", "gyt_trace_light_paths",
           "gyt_render_volume", "gyt_render_volume_device", "gyt_trace_volume_paths",
           "gyt_mesh_load_obj", "gyt_mesh_size", "gyt_mesh_read", "gyt_mesh_transform", "gyt_mesh_destroy",
           "gyt_render_device_noalloc", "gyt_context_set_batch_config", "gyt_context_get_batch_config",
           "gyt_render_batch_device", "gyt_render_batch", "gyt_batch_autotune", "gyt_scene_set_materials",
           "gyt_scene_freeze_sampling", "gyt_scene_read_wide_bvh", "gyt_bsdf_table",
           "gyt_diff_forward", "gyt_diff_backward", "gyt_diff_backward_paths"]

# BVH builders (GYT_BVH_BUILD_* in include/gyt.h)
BVH_BUILD_HOST = 0
BVH_BUILD_DEVICE = 1

# gyt_scene_set_materials flags
KEEP_LIGHT_SAMPLING = 1

# GytRenderParams.flags: HaltonSampler + HaltonEnum instead of Sobol' (GYT_SAMPLER_HALTON).
SAMPLER_HALTON = 1
SAMPLERS = {"sobol": 0, "halton": SAMPLER_HALTON}

# GytRenderParams.flags of the volumetric entry points: equi-angular sampling
# (VolPathTracing's equalAngular, GYT_VOLUME_EQUI_ANGULAR).
VOLUME_EQUI_ANGULAR = 2

# Path slots of the library's built-in scratch array (GYT_NOALLOC_MAX_PATHS in include/gyt.h).
NOALLOC_MAX_PATHS = 32768


class GytError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


class GytSceneDesc(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_uint32), ("n_triangles", ctypes.c_uint32), ("n_spheres", ctypes.c_uint32),
                ("n_materials", ctypes.c_uint32), ("n_emission", ctypes.c_uint32),
                ("vertices", ctypes.c_void_p), ("normals", ctypes.c_void_p), ("indices", ctypes.c_void_p),
                ("tri_material", ctypes.c_void_p), ("tri_emission", ctypes.c_void_p), ("spheres", ctypes.c_void_p),
                ("sphere_material", ctypes.c_void_p), ("mat_type", ctypes.c_void_p), ("mat_params", ctypes.c_void_p),
                ("emission", ctypes.c_void_p), ("env_w", ctypes.c_uint32), ("env_h", ctypes.c_uint32),
                ("env", ctypes.c_void_p), ("env_scale", ctypes.c_float), ("n_media", ctypes.c_uint32),
                ("media", ctypes.c_void_p), ("tri_medium", ctypes.c_void_p)]


class GytCamera(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_float * 3), ("look_at", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("fovy", ctypes.c_float), ("film_distance", ctypes.c_float), ("res_x", ctypes.c_uint32),
                ("res_y", ctypes.c_uint32)]


class GytRenderParams(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("rr_depth", ctypes.c_uint32),
                ("flags", ctypes.c_uint32)]


class GytRenderStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("path_slots", ctypes.c_uint64), ("iterations", ctypes.c_uint32),
                ("launches", ctypes.c_uint32), ("ms", ctypes.c_float)]


class GytProfile(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_float * 6), ("launches", ctypes.c_uint32 * 6), ("rays", ctypes.c_uint64 * 3),
                ("node_visits", ctypes.c_uint64 * 3), ("tri_tests", ctypes.c_uint64 * 3)]


class GytBatchConfig(ctypes.Structure):
    _fields_ = [("paths_in_flight", ctypes.c_uint32), ("stride_blocks_per_sm", ctypes.c_uint32),
                ("trace_blocks_per_sm", ctypes.c_uint32), ("use_graph", ctypes.c_uint32),
                ("bvh_width", ctypes.c_uint32)]


# profile slots (slot 4 is unused: the MIS rays are traced in the connect launch)
KERNELS = ["generate", "extend", "shade", "connect", "unused", "finish"]
TRAVERSALS = ["extend", "shadow", "mis"]


_lib = None


def load():
    """Load the native library (raises GytError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GytError(-1, "native library %s is missing; run gyunity_b200.build.build()" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P, U32, U64, I32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32
    L.gyt_context_create.argtypes = [I32, ctypes.POINTER(P)]
    L.gyt_context_destroy.argtypes = [P]
    L.gyt_context_destroy.restype = None
    L.gyt_last_error.argtypes = [P]
    L.gyt_last_error.restype = ctypes.c_char_p
    L.gyt_context_set_capacity.argtypes = [P, U32]
    L.gyt_context_set_profile.argtypes = [P, I32]
    L.gyt_profile_read.argtypes = [P, ctypes.POINTER(GytProfile)]
    L.gyt_context_set_bvh_width.argtypes = [P, I32]
    L.gyt_context_set_bvh_builder.argtypes = [P, I32]
    L.gyt_scene_read_bvh.argtypes = [P, P, U64, P, U64, ctypes.POINTER(U64)]
    L.gyt_scene_read_wide_bvh.argtypes = [P, P, U64, P, U64, ctypes.POINTER(U64)]
    L.gyt_scene_create.argtypes = [P, ctypes.POINTER(GytSceneDesc), ctypes.POINTER(P)]
    L.gyt_scene_destroy.argtypes = [P]
    L.gyt_scene_destroy.restype = None
    L.gyt_scene_info.argtypes = [P, P, P, P]
    L.gyt_render.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P]
    L.gyt_render_device.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P,
                                    ctypes.POINTER(GytRenderStats)]
    L.gyt_render_device_noalloc.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P, U32]
    L.gyt_trace_paths.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), U64, P, P, P, P,
                                  P, P]
    L.gyt_intersect.argtypes = [P, P, U64, P, I32, P, P, P, P]
    L.gyt_sobol.argtypes = [P, U64, P, P, P]
    L.gyt_sobol_enum_index.argtypes = [P, U32, U32, U64, P, P]
    L.gyt_halton.argtypes = [P, U64, P, P, P]
    L.gyt_halton_enum_index.argtypes = [P, U32, U32, U64, P, P]
    L.gyt_film_quantize.argtypes = [P, P, U32, U32, ctypes.c_float, P]
    L.gyt_film_save.argtypes = [P, P, U32, U32, ctypes.c_char_p]
    L.gyt_render_light_tracing.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P]
    L.gyt_render_light_tracing_device.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams),
                                                  P, ctypes.POINTER(GytRenderStats)]
    L.gyt_trace_light_paths.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), U64, P, P]
    L.gyt_render_volume.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P]
    L.gyt_render_volume_device.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P,
                                           ctypes.POINTER(GytRenderStats)]
    L.gyt_trace_volume_paths.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), U64, P,
                                         P, P]
    L.gyt_mesh_load_obj.argtypes = [ctypes.c_char_p, I32, ctypes.POINTER(P), ctypes.c_char_p, U32]
    L.gyt_mesh_size.argtypes = [P, ctypes.POINTER(U32)]
    L.gyt_mesh_read.argtypes = [P, P, P, P]
    L.gyt_mesh_transform.argtypes = [P, P, P, P]
    L.gyt_mesh_destroy.argtypes = [P]
    L.gyt_mesh_destroy.restype = None
    L.gyt_camera_raster_to_world.argtypes = [ctypes.POINTER(GytCamera), P]
    L.gyt_scene_set_materials.argtypes = [P, P, P, U32]
    L.gyt_scene_freeze_sampling.argtypes = [P, P]
    L.gyt_bsdf_table.argtypes = [P, U64, P, P, P, P]
    L.gyt_diff_forward.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P, P,
                                   ctypes.POINTER(GytRenderStats)]
    L.gyt_diff_backward.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), P, P, P, P, P,
                                    ctypes.POINTER(GytRenderStats)]
    L.gyt_diff_backward_paths.argtypes = [P, P, ctypes.POINTER(GytCamera), ctypes.POINTER(GytRenderParams), U64, P,
                                          P, P, P, P]
    L.gyt_context_set_batch_config.argtypes = [P, ctypes.POINTER(GytBatchConfig)]
    L.gyt_context_get_batch_config.argtypes = [P, ctypes.POINTER(GytBatchConfig)]
    L.gyt_render_batch_device.argtypes = [P, U32, P, P, P, P, ctypes.POINTER(GytRenderStats)]
    L.gyt_render_batch.argtypes = [P, U32, P, P, P, P]
    L.gyt_batch_autotune.argtypes = [P, U32, P, P, P, P, U32, ctypes.POINTER(GytBatchConfig),
                                     ctypes.POINTER(ctypes.c_float)]
    for name in EXPORTS:
        f = getattr(L, name)
        if f.restype is ctypes.c_int:  # default
            f.restype = I32
    _lib = L
    return L


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def camera_struct(cam):
    c = GytCamera()
    c.pos[:] = [float(v) for v in cam.pos]
    c.look_at[:] = [float(v) for v in cam.look_at]
    c.up[:] = [float(v) for v in cam.up]
    c.fovy = cam.fovy
    c.film_distance = cam.film_distance
    c.res_x = cam.res_x
    c.res_y = cam.res_y
    return c


def params_struct(p):
    flags = SAMPLERS[getattr(p, "sampler", "sobol")]
    if getattr(p, "equi_angular", False):
        flags |= VOLUME_EQUI_ANGULAR
    return GytRenderParams(p.spp, p.max_depth, p.rr_depth, flags)


def scene_struct(sd):
    """Build a GytSceneDesc pointing into contiguous copies of the arrays;
    returns (struct, keep-alive list)."""
    def c(a, dt):
        return None if a is None else np.ascontiguousarray(a, dt)
    keep = [c(sd.vertices, np.float32), c(sd.normals, np.float32), c(sd.indices, np.uint32),
            c(sd.tri_material, np.uint32), c(sd.tri_emission, np.int32), c(sd.spheres, np.float32),
            c(sd.sphere_material, np.uint32), c(sd.mat_type, np.uint32), c(sd.mat_params, np.float32),
            c(sd.emission, np.float32), c(sd.env, np.float32), c(getattr(sd, "media", None), np.float32),
            c(getattr(sd, "tri_medium", None), np.int32)]
    s = GytSceneDesc()
    s.n_vertices, s.n_triangles = sd.vertices.shape[0], sd.n_triangles
    s.n_spheres, s.n_materials, s.n_emission = sd.n_spheres, sd.mat_type.shape[0], sd.emission.shape[0]
    (s.vertices, s.normals, s.indices, s.tri_material, s.tri_emission, s.spheres, s.sphere_material, s.mat_type,
     s.mat_params, s.emission) = [None if a is None else a.ctypes.data for a in keep[:10]]
    if sd.env is not None:
        s.env_h, s.env_w = sd.env.shape[:2]
        s.env = keep[10].ctypes.data
    s.env_scale = sd.env_scale
    if keep[11] is not None:
        s.n_media = keep[11].reshape(-1, 7).shape[0]
        s.media = keep[11].ctypes.data
    if keep[12] is not None:
        s.tri_medium = keep[12].ctypes.data
    return s, keep
