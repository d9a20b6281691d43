"""Meshes from Wavefront OBJ files and their placement in a scene.

``Mesh.load_obj`` is Mesh::LoadFromFile (mesh/Mesh.cpp:7-90) through the
library (gyt_mesh_load_obj); ``Mesh.transform`` is the per-triangle
Triangle::SetTransform of Scene::AddMesh (visual/Scene.h:68-77) on the GPU
(gyt_mesh_transform); ``add_mesh`` appends the triangles to a SceneDesc with
one material, as Scene::AddPrimitive does for each of them.

``Transform`` builds the matrices as math/Transform.cpp does, in float32 and
in the reference's operation order (a matrix times a vector is the sum of its
columns from the last: ((c3 v3 + c2 v2) + c1 v1) + c0 v0), so that a composed
transform has the reference's bits.
"""
import ctypes
import ctypes.util

import numpy as np

from . import _capi as _c
from ._capi import GytError

_F = np.float32
# PI and Radians (common/Core.h:185, math/MathUtils.h:63), in float
_PI = _F(3.14159265358979)
_libm = None


def _sincos(theta_deg):
    """std::sin / std::cos of Radians(theta) in float, through the C
    library's sinf and cosf as the reference calls them."""
    global _libm
    if _libm is None:
        _libm = ctypes.CDLL(ctypes.util.find_library("m"))
        for f in (_libm.sinf, _libm.cosf):
            f.argtypes = [ctypes.c_float]
            f.restype = ctypes.c_float
    r = _F(_PI / _F(180)) * _F(theta_deg)
    return _F(_libm.sinf(float(r))), _F(_libm.cosf(float(r)))


def _mat_vec(a, v):
    """Matrix4 * Vector4 (math/Linagl.h:936-947): columns from the last."""
    r = a[:, 3] * v[3]
    r = a[:, 2] * v[2] + r
    r = a[:, 1] * v[1] + r
    return a[:, 0] * v[0] + r


def _mat_mul(a, b):
    """Matrix4 * Matrix4: column i is a * (column i of b)."""
    out = np.empty((4, 4), _F)
    for i in range(4):
        out[:, i] = _mat_vec(a, b[:, i])
    return out


class Transform:
    """Transform (math/Transform.h): a 4x4 float32 matrix and its inverse."""

    def __init__(self, m=None, inv=None):
        self.m = np.eye(4, dtype=_F) if m is None else np.asarray(m, _F).reshape(4, 4)
        self.inv = np.eye(4, dtype=_F) if inv is None else np.asarray(inv, _F).reshape(4, 4)

    @staticmethod
    def Translate(v):
        m, inv = np.eye(4, dtype=_F), np.eye(4, dtype=_F)
        m[:3, 3] = np.asarray(v, _F)
        inv[:3, 3] = -np.asarray(v, _F)
        return Transform(m, inv)

    @staticmethod
    def Scale(sx, sy, sz):
        s = np.array([sx, sy, sz], _F)
        m, inv = np.eye(4, dtype=_F), np.eye(4, dtype=_F)
        m[[0, 1, 2], [0, 1, 2]] = s
        inv[[0, 1, 2], [0, 1, 2]] = _F(1) / s
        return Transform(m, inv)

    @staticmethod
    def _rot(theta, axes):
        s, c = _sincos(theta)
        i, j = axes
        m = np.eye(4, dtype=_F)
        m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
        return Transform(m, m.T.copy())

    @staticmethod
    def RotateX(theta):
        return Transform._rot(theta, (1, 2))

    @staticmethod
    def RotateY(theta):
        s, c = _sincos(theta)
        m = np.eye(4, dtype=_F)
        m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
        return Transform(m, m.T.copy())

    @staticmethod
    def RotateZ(theta):
        return Transform._rot(theta, (0, 1))

    def __mul__(self, t):
        """Transform::operator* (math/Transform.h:253-255)."""
        return Transform(_mat_mul(self.m, t.m), _mat_mul(t.inv, self.inv))


class Mesh:
    """A loaded OBJ mesh: one record of three vertices per triangle."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load_obj(cls, path, reverse_vertices=False):
        L = _c.load()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = L.gyt_mesh_load_obj(str(path).encode(), 1 if reverse_vertices else 0, ctypes.byref(h), err, 512)
        if rc:
            raise GytError(rc, "mesh_load_obj: " + err.value.decode(errors="replace"))
        return cls(h)

    @property
    def n_triangles(self):
        n = ctypes.c_uint32()
        _c.load().gyt_mesh_size(self._h, ctypes.byref(n))
        return n.value

    def arrays(self):
        """positions (n, 3, 3), normals (n, 3, 3), uvs (n, 3, 2), float32."""
        n = self.n_triangles
        p = np.empty((n, 3, 3), _F)
        nr = np.empty((n, 3, 3), _F)
        uv = np.empty((n, 3, 2), _F)
        _c.load().gyt_mesh_read(self._h, _c.ptr(p), _c.ptr(nr), _c.ptr(uv))
        return p, nr, uv

    def transform(self, t, ctx=None):
        """Triangle::SetTransform of every triangle, on the GPU of ctx."""
        from . import default_context
        ctx = ctx or default_context()
        m = np.ascontiguousarray(t.m, _F)
        inv = np.ascontiguousarray(t.inv, _F)
        ctx.check(ctx._lib.gyt_mesh_transform(ctx.handle, self._h, _c.ptr(m), _c.ptr(inv)))
        return self

    def close(self):
        if self._h:
            _c.load().gyt_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def add_mesh(sd, mesh, mat_type, mat_params, emission=None):
    """A copy of SceneDesc sd with the mesh's triangles added after its own,
    all with one new material (GYT_MAT_* type and 16 parameters) and, with
    emission (RGB), as one area light each (Scene::AddMesh + AddPrimitive)."""
    import dataclasses
    p, n, _ = mesh.arrays()
    nt = p.shape[0]
    nv0 = sd.vertices.shape[0]
    normals = sd.normals if sd.normals is not None else np.zeros((nv0, 3), _F)
    mid = sd.mat_type.shape[0]
    em = sd.emission
    tri_em = np.full(nt, -1, np.int32)
    if emission is not None:
        tri_em[:] = em.shape[0]
        em = np.concatenate([em, np.asarray(emission, _F).reshape(1, 3)])
    return dataclasses.replace(
        sd,
        vertices=np.concatenate([sd.vertices, p.reshape(-1, 3)]).astype(_F),
        normals=np.concatenate([normals, n.reshape(-1, 3)]).astype(_F),
        indices=np.concatenate([sd.indices, (nv0 + np.arange(3 * nt, dtype=np.uint32)).reshape(nt, 3)]).astype(
            np.uint32),
        tri_material=np.concatenate([sd.tri_material, np.full(nt, mid, np.uint32)]),
        tri_emission=np.concatenate([sd.tri_emission, tri_em]),
        mat_type=np.concatenate([sd.mat_type, np.array([mat_type], np.uint32)]),
        mat_params=np.concatenate([sd.mat_params, np.asarray(mat_params, _F).reshape(1, 16)]),
        emission=em)
