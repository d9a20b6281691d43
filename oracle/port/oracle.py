"""ctypes wrapper of the CPU restatement (oracle/port/pt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path. Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "pt_oracle.cpp")
LIB = os.path.join(HERE, "libgyoracle.so")
TABLES = os.path.join(HERE, "..", "..", "gyunity_b200", "_gen", "sobol_tables.h")


def build(force=False):
    """Compile the restatement with g++ (unfused FP like the reference build)."""
    if os.path.exists(LIB) and not force and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                                                          os.path.getmtime(TABLES)):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", SRC, "-o", LIB]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout[-3000:])
    return LIB


class SceneIn(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_uint32), ("n_triangles", ctypes.c_uint32), ("n_spheres", ctypes.c_uint32),
                ("n_materials", ctypes.c_uint32), ("n_emission", ctypes.c_uint32),
                ("vertices", ctypes.c_void_p), ("normals", ctypes.c_void_p), ("indices", ctypes.c_void_p),
                ("tri_material", ctypes.c_void_p), ("tri_emission", ctypes.c_void_p), ("spheres", ctypes.c_void_p),
                ("sphere_material", ctypes.c_void_p), ("mat_type", ctypes.c_void_p), ("mat_params", ctypes.c_void_p),
                ("emission", ctypes.c_void_p), ("env_w", ctypes.c_uint32), ("env_h", ctypes.c_uint32),
                ("env", ctypes.c_void_p), ("env_scale", ctypes.c_float)]


class CameraIn(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_float * 3), ("look_at", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("fovy", ctypes.c_float), ("film_distance", ctypes.c_float), ("res_x", ctypes.c_uint32),
                ("res_y", ctypes.c_uint32)]


class ParamsIn(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("rr_depth", ctypes.c_uint32),
                ("sampler", ctypes.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        L.gyo_tables_digest.restype = ctypes.c_char_p
        L.gyo_sobol.restype = ctypes.c_float
        L.gyo_sobol.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
        L.gyo_enum_index.restype = ctypes.c_uint64
        L.gyo_enum_index.argtypes = [ctypes.c_uint32] * 5
        L.gyo_halton.restype = ctypes.c_float
        L.gyo_halton.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
        L.gyo_halton_enum_index.restype = ctypes.c_uint64
        L.gyo_halton_enum_index.argtypes = [ctypes.c_uint32] * 5
        L.gyo_raster_to_world.argtypes = [ctypes.POINTER(CameraIn), ctypes.c_void_p]
        L.gyo_scene_create.restype = ctypes.c_void_p
        L.gyo_scene_create.argtypes = [ctypes.POINTER(SceneIn)]
        L.gyo_scene_destroy.argtypes = [ctypes.c_void_p]
        L.gyo_closest_hit.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_any_hit.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_paths.argtypes = [ctypes.c_void_p, ctypes.POINTER(CameraIn), ctypes.POINTER(ParamsIn), ctypes.c_int64,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_set_trace.argtypes = [ctypes.c_int]
        L.gyo_render.argtypes = [ctypes.c_void_p, ctypes.POINTER(CameraIn), ctypes.POINTER(ParamsIn),
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.gyo_bsdf.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_adjoint.argtypes = [ctypes.c_void_p, ctypes.POINTER(CameraIn), ctypes.POINTER(ParamsIn), ctypes.c_int64,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_set_sampling_materials.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_ggx_dlog_alpha.restype = ctypes.c_double
        L.gyo_ggx_dlog_alpha.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        L.gyo_ggx_log_f.restype = ctypes.c_double
        L.gyo_ggx_log_f.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def camera_in(cam):
    c = CameraIn()
    c.pos[:] = list(cam.pos)
    c.look_at[:] = list(cam.look_at)
    c.up[:] = list(cam.up)
    c.fovy = cam.fovy
    c.film_distance = cam.film_distance
    c.res_x = cam.res_x
    c.res_y = cam.res_y
    return c


SAMPLERS = {"sobol": 0, "halton": 1}


def params_in(p):
    return ParamsIn(p.spp, p.max_depth, p.rr_depth, SAMPLERS[getattr(p, "sampler", "sobol")])


class OracleScene:
    """The oracle's own copy of a SceneDesc (FP32 and FP64 versions)."""

    def __init__(self, sd):
        self.sd = sd
        self._keep = [np.ascontiguousarray(a) if a is not None else None for a in (
            sd.vertices.astype(np.float32), None if sd.normals is None else sd.normals.astype(np.float32),
            sd.indices.astype(np.uint32), sd.tri_material.astype(np.uint32), sd.tri_emission.astype(np.int32),
            None if sd.spheres is None else sd.spheres.astype(np.float32),
            None if sd.sphere_material is None else sd.sphere_material.astype(np.uint32),
            sd.mat_type.astype(np.uint32), sd.mat_params.astype(np.float32), sd.emission.astype(np.float32),
            None if sd.env is None else sd.env.astype(np.float32))]
        k = self._keep
        s = SceneIn()
        s.n_vertices, s.n_triangles = sd.vertices.shape[0], sd.n_triangles
        s.n_spheres, s.n_materials, s.n_emission = sd.n_spheres, sd.mat_type.shape[0], sd.emission.shape[0]
        (s.vertices, s.normals, s.indices, s.tri_material, s.tri_emission, s.spheres, s.sphere_material,
         s.mat_type, s.mat_params, s.emission) = [_p(a) for a in k[:10]]
        s.env_h, s.env_w = (0, 0) if sd.env is None else sd.env.shape[:2]
        s.env = _p(k[10])
        s.env_scale = sd.env_scale
        self.handle = lib().gyo_scene_create(ctypes.byref(s))

    def close(self):
        if self.handle:
            lib().gyo_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def closest_hit(self, rays, precision=64):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 7)
        n = rays.shape[0]
        prim = np.empty(n, np.int32)
        t, b1, b2 = (np.empty(n, np.float64) for _ in range(3))
        lib().gyo_closest_hit(self.handle, n, _p(rays), precision, _p(prim), _p(t), _p(b1), _p(b2))
        return prim, t, b1, b2

    def any_hit(self, rays):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 7)
        out = np.empty(rays.shape[0], np.int32)
        lib().gyo_any_hit(self.handle, rays.shape[0], _p(rays), _p(out))
        return out.astype(bool)

    def paths(self, x, y, s, precision=64, threads=0, camera=None, params=None, force_rr=None, return_rr=False,
              force_occ=None, force_mis=None, return_decisions=False):
        """Radiance of paths (x, y, s). ``force_rr``/``force_occ``/``force_mis``
        replay recorded decisions (bit i = bounce i): a roulette number was
        drawn, the shadow ray was occluded, the MIS ray reached the light."""
        x, y, s = (np.ascontiguousarray(np.asarray(a, np.uint32)) for a in (x, y, s))
        n = x.shape[0]
        L = np.empty((n, 3), np.float64)
        cur = np.empty(n, np.int32)
        rr, occ, mis = (np.empty(n, np.uint64) for _ in range(3))
        f = [None if a is None else np.ascontiguousarray(np.asarray(a, np.uint64)) for a in (force_rr, force_occ,
                                                                                           force_mis)]
        c = camera_in(camera or self.sd.camera)
        p = params_in(params or self.sd.params)
        lib().gyo_paths(self.handle, ctypes.byref(c), ctypes.byref(p), n, _p(x), _p(y), _p(s), precision, _p(L),
                        _p(cur), threads, _p(f[0]), _p(rr), _p(f[1]), _p(f[2]), _p(occ), _p(mis))
        if return_decisions:
            return L, cur, rr, occ, mis
        return (L, cur, rr) if return_rr else (L, cur)

    def adjoint(self, x, y, s, delta, precision=64, threads=0, camera=None, params=None, force_rr=None,
                force_occ=None, force_mis=None):
        """Path replay adjoint of paths (x, y, s) with adjoint weights delta
        (n, 3), replaying the given decisions. Returns the gradient sums per
        material (n_materials, 4: a.r, a.g, a.b, alpha) and per emission row
        (n_emission, 3), and the path radiance (n, 3)."""
        x, y, s = (np.ascontiguousarray(np.asarray(a, np.uint32)) for a in (x, y, s))
        n = x.shape[0]
        d = np.ascontiguousarray(delta, np.float32).reshape(n, 3)
        nm, ne = int(self.sd.mat_type.shape[0]), int(self.sd.emission.shape[0])
        gm = np.zeros((nm, 4), np.float64)
        ge = np.zeros((max(ne, 1), 3), np.float64)
        L = np.empty((n, 3), np.float64)
        f = [None if a is None else np.ascontiguousarray(np.asarray(a, np.uint64)) for a in (force_rr, force_occ,
                                                                                           force_mis)]
        c = camera_in(camera or self.sd.camera)
        p = params_in(params or self.sd.params)
        lib().gyo_adjoint(self.handle, ctypes.byref(c), ctypes.byref(p), n, _p(x), _p(y), _p(s), precision, _p(d),
                          threads, _p(f[0]), _p(f[1]), _p(f[2]), nm, ne, _p(gm), _p(ge), _p(L))
        return gm, ge[:ne], L

    def set_sampling_materials(self, mat_params=None):
        """Test hook: sample BSDFs (and their pdfs) with these parameters
        while evaluating them with the scene's (None restores the scene's)."""
        self._smp = None if mat_params is None else np.ascontiguousarray(mat_params, np.float32)
        lib().gyo_set_sampling_materials(self.handle, _p(self._smp))

    def render(self, rows=None, precision=64, threads=0, camera=None, params=None):
        cam = camera or self.sd.camera
        c = camera_in(cam)
        p = params_in(params or self.sd.params)
        film = np.zeros((cam.res_y, cam.res_x, 4), np.float64)
        r0, r1 = (0, cam.res_y) if rows is None else rows
        lib().gyo_render(self.handle, ctypes.byref(c), ctypes.byref(p), r0, r1, precision, _p(film), threads)
        return film


def ggx_dlog_alpha(alpha, wo, wi):
    """d log f / d alpha of the GGX reflection lobe (local directions)."""
    a, b = np.ascontiguousarray(wo, np.float64), np.ascontiguousarray(wi, np.float64)
    return lib().gyo_ggx_dlog_alpha(float(alpha), _p(a), _p(b))


def ggx_log_f(alpha, wo, wi):
    """log of the GGX reflection lobe's value (eta = k = 1.5, a = 1)."""
    a, b = np.ascontiguousarray(wo, np.float64), np.ascontiguousarray(wi, np.float64)
    return lib().gyo_ggx_log_f(float(alpha), _p(a), _p(b))


def sobol(dims, indices):
    L = lib()
    return np.array([L.gyo_sobol(int(d), int(i)) for d, i in zip(dims, indices)], np.float32)


def enum_index(res_x, res_y, s, x, y):
    L = lib()
    return np.array([L.gyo_enum_index(res_x, res_y, int(a), int(b), int(c)) for a, b, c in zip(s, x, y)], np.uint64)


def halton(dims, indices):
    """HaltonSampler (Faure permutations) for (dim, index) pairs."""
    L = lib()
    return np.array([L.gyo_halton(int(d), int(i)) for d, i in zip(dims, indices)], np.float32)


def halton_enum_index(res_x, res_y, s, x, y):
    L = lib()
    return np.array([L.gyo_halton_enum_index(res_x, res_y, int(a), int(b), int(c)) for a, b, c in zip(s, x, y)],
                    np.uint64)


def raster_to_world(cam):
    out = np.empty(16, np.float64)
    c = camera_in(cam)
    lib().gyo_raster_to_world(ctypes.byref(c), _p(out))
    return out.reshape(4, 4)


def bsdf_table(cases):
    out = np.empty((cases.shape[0], 11), np.float64)
    lib().gyo_bsdf(cases.shape[0], _p(np.ascontiguousarray(cases)), _p(out))
    return out
