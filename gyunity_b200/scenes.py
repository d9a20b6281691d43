"""Seeded procedural scenes for the path tracing workloads.

A ``SceneDesc`` is the flat, array-only description that crosses the C ABI
(``GytSceneDesc`` in include/gyt.h). It follows the reference's scene model:

* primitives are triangles (``shape/Triangle.h``) followed by analytic spheres
  (``shape/Sphere.h``); the primitive id of triangle ``t`` is ``t`` and of
  sphere ``s`` is ``n_triangles + s`` (the order ``Scene::AddPrimitive`` hands
  out ids in, ``visual/Scene.h:49-58``);
* every emitting triangle is its own ``AreaLight`` (``light/AreaLight.h``) and
  the light list is the emitting triangles in triangle order, then the
  environment light if there is one (``Scene::AddLight``, ``visual/Scene.h:60``);
* per-vertex shading normals are interpolated as in
  ``Triangle::QueryIntersectionInfo`` (``shape/Triangle.cpp:37-38``); without
  them the face normal ``Cross(p1-p0, p2-p0).Norm()`` is used at every corner.

Material records (type, 16 floats):

====  ======================  ===========================================
type  reference material      params used
====  ======================  ===========================================
0     DiffuseMaterial         [0:3] kd
1     MirrorMaterial          [0:3] kr
2     GlassMaterial           [0:3] kr, [3:6] kt, [15] eta1, [8] eta2
3     GGX conductor           [0:3] R, [6] alpha_x, [7] alpha_y,
      (RoughnessMaterial)     [9:12] eta, [12:15] k
4     GGX rough dielectric    [0:3] kr, [3:6] kt, [6] alpha_x, [7] alpha_y,
      (RoughDielectricMat.)   [8] eta
====  ======================  ===========================================

Alpha is stored directly; ``roughness_to_alpha`` converts a reference
roughness value (``visual/Microfacet.h:49-54``) when a caller has one.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

MAT_DIFFUSE, MAT_MIRROR, MAT_GLASS, MAT_CONDUCTOR, MAT_DIELECTRIC, MAT_NONE = 0, 1, 2, 3, 4, 5

# fovy of the reference's Cornell-box camera (Gyunity_exe/main.cpp:712)
CORNELL_FOVY = 53.13010235415597


@dataclasses.dataclass
class Camera:
    pos: tuple = (0.0, 0.0, 3.0)
    look_at: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    fovy: float = CORNELL_FOVY
    film_distance: float = 1.0
    res_x: int = 256
    res_y: int = 256


@dataclasses.dataclass
class RenderParams:
    spp: int = 16
    max_depth: int = 8
    rr_depth: int = 5   # Russian roulette applies when bounce index i > rr_depth (reference: 5)
    sampler: str = "sobol"  # "sobol" (SobolSampler + SobolEnum) or "halton" (HaltonSampler + HaltonEnum)
    equi_angular: bool = False  # volumetric renders: VolPathTracing's equalAngular (GYT_VOLUME_EQUI_ANGULAR)


@dataclasses.dataclass
class SceneDesc:
    vertices: np.ndarray                 # (nv, 3) float32
    indices: np.ndarray                  # (nt, 3) uint32
    tri_material: np.ndarray             # (nt,) uint32
    tri_emission: np.ndarray             # (nt,) int32, -1 = not a light
    mat_type: np.ndarray                 # (nm,) uint32
    mat_params: np.ndarray               # (nm, 16) float32
    emission: np.ndarray                 # (ne, 3) float32
    normals: Optional[np.ndarray] = None  # (nv, 3) float32
    spheres: Optional[np.ndarray] = None  # (ns, 4) float32: cx, cy, cz, r
    sphere_material: Optional[np.ndarray] = None  # (ns,) uint32
    env: Optional[np.ndarray] = None     # (h, w, 3) float32, row 0 = top (theta = 0)
    env_scale: float = 1.0
    media: Optional[np.ndarray] = None   # (nmed, 7) float32: sigma_a rgb, sigma_s rgb, HG g
    tri_medium: Optional[np.ndarray] = None  # (nt, 2) int32: medium inside, outside (-1 none)
    camera: Camera = dataclasses.field(default_factory=Camera)
    params: RenderParams = dataclasses.field(default_factory=RenderParams)
    name: str = ""

    @property
    def n_triangles(self) -> int:
        return int(self.indices.shape[0])

    @property
    def n_spheres(self) -> int:
        return 0 if self.spheres is None else int(self.spheres.shape[0])

    def n_paths(self) -> int:
        return self.camera.res_x * self.camera.res_y * self.params.spp


def roughness_to_alpha(roughness: float) -> float:
    """``GGXDistribution::RoughnessToAlpha`` (visual/Microfacet.h:49-54) in float32."""
    r = np.float32(max(roughness, 1e-3))
    x = np.float32(math.log(r))
    return float(np.float32(1.62142) + np.float32(0.819955) * x + np.float32(0.1734) * x * x
                 + np.float32(0.0171201) * x * x * x + np.float32(0.000640711) * x * x * x * x)


def _mat(kind, a=(0, 0, 0), b=(0, 0, 0), ax=0.0, ay=0.0, eta=1.5, ceta=(1.5, 1.5, 1.5), k=(1.5, 1.5, 1.5), eta1=1.0):
    p = np.zeros(16, np.float32)
    p[0:3] = a
    p[3:6] = b
    p[6] = ax
    p[7] = ay
    p[8] = eta
    p[9:12] = ceta
    p[12:15] = k
    p[15] = eta1
    return kind, p


class _Builder:
    def __init__(self):
        self.v, self.n, self.i, self.tm, self.te = [], [], [], [], []
        self.mt, self.mp, self.em = [], [], []
        self.nv = 0

    def material(self, kind, p) -> int:
        self.mt.append(kind)
        self.mp.append(p)
        return len(self.mt) - 1

    def quad(self, p0, p1, p2, p3, normal, mat, emission=None):
        """Two triangles (p0,p1,p2) and (p2,p3,p0) as the reference fixture
        (Gyunity_exe/CornellBox.h:437-440) with a constant shading normal."""
        base = self.nv
        self.v.append(np.array([p0, p1, p2, p3], np.float32))
        self.n.append(np.array([normal] * 4, np.float32))
        self.nv += 4
        self.i.append(np.array([[base, base + 1, base + 2], [base + 2, base + 3, base]], np.uint32))
        self.tm += [mat, mat]
        if emission is None:
            self.te += [-1, -1]
        else:
            e = len(self.em)
            self.em.append(emission)
            self.em.append(emission)
            self.te += [e, e + 1]

    def tris(self, verts, normals, idx, mats):
        self.v.append(verts.astype(np.float32))
        self.n.append(normals.astype(np.float32))
        self.i.append(idx.astype(np.uint32) + np.uint32(self.nv))
        self.nv += verts.shape[0]
        self.tm += list(np.asarray(mats, np.uint32))
        self.te += [-1] * idx.shape[0]

    def build(self, **kw) -> SceneDesc:
        return SceneDesc(
            vertices=np.ascontiguousarray(np.concatenate(self.v).astype(np.float32)),
            normals=np.ascontiguousarray(np.concatenate(self.n).astype(np.float32)),
            indices=np.ascontiguousarray(np.concatenate(self.i).astype(np.uint32)),
            tri_material=np.asarray(self.tm, np.uint32),
            tri_emission=np.asarray(self.te, np.int32),
            mat_type=np.asarray(self.mt, np.uint32),
            mat_params=np.ascontiguousarray(np.stack(self.mp).astype(np.float32)),
            emission=np.asarray(self.em, np.float32).reshape(-1, 3),
            **kw)


def _cornell_walls(b: _Builder, light_radiance=(12.0, 12.0, 12.0), light_half=0.25, light=True):
    """The +-1 Cornell box of CornellBoxMesh (Gyunity_exe/CornellBox.h:402-591):
    left red, right blue, back/floor/ceiling grey 0.75, and (``light``) a
    ceiling light quad at y = 0.965 facing -y. Returns nothing; appends 10
    wall triangles and 2 light triangles."""
    grey = b.material(*_mat(MAT_DIFFUSE, (0.75, 0.75, 0.75)))
    red = b.material(*_mat(MAT_DIFFUSE, (0.75, 0.25, 0.25)))
    blue = b.material(*_mat(MAT_DIFFUSE, (0.25, 0.25, 0.75)))
    black = b.material(*_mat(MAT_DIFFUSE, (0.0, 0.0, 0.0)))
    p = [(-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (1, -1, 1), (1, -1, -1), (1, 1, -1), (1, 1, 1)]
    b.quad(p[0], p[1], p[2], p[3], (1, 0, 0), red)
    # right wall: triangles (p4,p5,p6) and (p4,p6,p7) in the fixture
    base = b.nv
    b.v.append(np.array([p[4], p[5], p[6], p[7]], np.float32))
    b.n.append(np.array([(-1, 0, 0)] * 4, np.float32))
    b.nv += 4
    b.i.append(np.array([[base, base + 1, base + 2], [base, base + 2, base + 3]], np.uint32))
    b.tm += [blue, blue]
    b.te += [-1, -1]
    # back (p1,p5,p6),(p1,p6,p2); floor (p0,p4,p5),(p0,p5,p1); ceiling (p3,p7,p6),(p3,p6,p2)
    for (q0, q1, q2, q3), nrm in (((1, 5, 6, 2), (0, 0, 1)), ((0, 4, 5, 1), (0, 1, 0)), ((3, 7, 6, 2), (0, -1, 0))):
        base = b.nv
        b.v.append(np.array([p[q0], p[q1], p[q2], p[q3]], np.float32))
        b.n.append(np.array([nrm] * 4, np.float32))
        b.nv += 4
        b.i.append(np.array([[base, base + 1, base + 2], [base, base + 2, base + 3]], np.uint32))
        b.tm += [grey, grey]
        b.te += [-1, -1]
    if not light:
        return
    h = light_half
    l0, l1, l2, l3 = (h, 0.965, h), (h, 0.965, -h), (-h, 0.965, -h), (-h, 0.965, h)
    base = b.nv
    b.v.append(np.array([l0, l1, l2, l3], np.float32))
    b.n.append(np.array([(0, -1, 0)] * 4, np.float32))
    b.nv += 4
    b.i.append(np.array([[base, base + 1, base + 2], [base, base + 2, base + 3]], np.uint32))
    b.tm += [black, black]
    e = len(b.em)
    b.em += [light_radiance, light_radiance]
    b.te += [e, e + 1]


def cornell_box(res=256, spp=16, max_depth=8, rr_depth=3, spheres=True) -> SceneDesc:
    """Cornell box, plain path tracing: 10 wall triangles, a 0.5 x 0.5 ceiling
    light (radiance 12), a mirror and a glass (IOR 1.5) sphere of radius 0.4."""
    b = _Builder()
    _cornell_walls(b)
    kw = {}
    if spheres:
        mirror = b.material(*_mat(MAT_MIRROR, (1, 1, 1)))
        glass = b.material(*_mat(MAT_GLASS, (1, 1, 1), (1, 1, 1), eta=1.5, eta1=1.0))
        kw["spheres"] = np.array([[-0.5, -0.6, -0.3, 0.4], [0.5, -0.6, 0.3, 0.4]], np.float32)
        kw["sphere_material"] = np.array([mirror, glass], np.uint32)
    return b.build(camera=Camera(res_x=res, res_y=res), params=RenderParams(spp, max_depth, rr_depth),
                   name="cornell_box_%dx%d_%dspp" % (res, res, spp), **kw)


def cornell_fog(res=128, spp=8, max_depth=8, sigma_a=0.05, sigma_s=0.5, g=0.3, spheres=True) -> SceneDesc:
    """CornellBoxMedium (Gyunity_exe/CornellBox.h:1631-1700): the Cornell box
    filled with one homogeneous medium, closed at z = 1 by a front quad of no
    material whose MediumInterface is (inside: the medium, outside: none);
    the walls keep the ray's medium. The reference's medium is sigma_s = 1,
    sigma_a = 0, g = 0; here thinner and forward-scattering, with the
    mirror and glass spheres of cornell_box."""
    sd = cornell_box(res=res, spp=spp, max_depth=max_depth, rr_depth=5, spheres=spheres)
    nv = sd.vertices.shape[0]
    front = np.array([[-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float32)
    none = sd.mat_type.shape[0]
    nt = sd.n_triangles
    tri_medium = np.full((nt + 2, 2), -1, np.int32)
    tri_medium[nt:] = (0, -1)
    return dataclasses.replace(
        sd,
        vertices=np.concatenate([sd.vertices, front]),
        normals=np.concatenate([sd.normals, np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))]),
        indices=np.concatenate([sd.indices, np.array([[nv, nv + 1, nv + 2], [nv, nv + 2, nv + 3]], np.uint32)]),
        tri_material=np.concatenate([sd.tri_material, np.array([none, none], np.uint32)]),
        tri_emission=np.concatenate([sd.tri_emission, np.array([-1, -1], np.int32)]),
        mat_type=np.concatenate([sd.mat_type, np.array([MAT_NONE], np.uint32)]),
        mat_params=np.concatenate([sd.mat_params, np.zeros((1, 16), np.float32)]),
        media=np.array([[sigma_a] * 3 + [sigma_s] * 3 + [g]], np.float32),
        tri_medium=tri_medium,
        name="cornell_fog_%dx%d_%dspp" % (res, res, spp))


def fog_ball_box(res=48, spp=4, max_depth=6, level=2, sigma_a=0.1, sigma_s=2.0, g=0.5) -> SceneDesc:
    """The Cornell box (no spheres, no fog in the box) holding a ball of fog:
    a level-``level`` icosphere of radius 0.45 at (0, -0.45, 0) with no
    material whose MediumInterface is (inside: the medium, outside: none),
    outward normals. Camera rays and light paths enter and leave the medium
    through it repeatedly; shadow rays cross it."""
    sd = cornell_box(res=res, spp=spp, max_depth=max_depth, rr_depth=5, spheres=False)
    v, f = icosphere(level)
    nv = sd.vertices.shape[0]
    none = sd.mat_type.shape[0]
    nt = sd.n_triangles
    ball = (v * 0.45 + np.array([0.0, -0.45, 0.0])).astype(np.float32)
    tri_medium = np.full((nt + f.shape[0], 2), -1, np.int32)
    tri_medium[nt:] = (0, -1)
    return dataclasses.replace(
        sd,
        vertices=np.concatenate([sd.vertices, ball]),
        normals=np.concatenate([sd.normals, v.astype(np.float32)]),
        indices=np.concatenate([sd.indices, (f + nv).astype(np.uint32)]),
        tri_material=np.concatenate([sd.tri_material, np.full(f.shape[0], none, np.uint32)]),
        tri_emission=np.concatenate([sd.tri_emission, np.full(f.shape[0], -1, np.int32)]),
        mat_type=np.concatenate([sd.mat_type, np.array([MAT_NONE], np.uint32)]),
        mat_params=np.concatenate([sd.mat_params, np.zeros((1, 16), np.float32)]),
        media=np.array([[sigma_a] * 3 + [sigma_s] * 3 + [g]], np.float32),
        tri_medium=tri_medium,
        name="fog_ball_box_%dx%d_%dspp" % (res, res, spp))


# ---------------------------------------------------------------- meshes ----

def _hash3(ix, iy, iz, seed):
    """Integer lattice hash -> float in [-1, 1] (xorshift-multiply mix)."""
    h = (ix.astype(np.uint64) * np.uint64(0x8DA6B343) ^ iy.astype(np.uint64) * np.uint64(0xD8163841)
         ^ iz.astype(np.uint64) * np.uint64(0xCB1AB31F) ^ np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15))
    h ^= h >> np.uint64(31)
    h *= np.uint64(0xBF58476D1CE4E5B9)
    h ^= h >> np.uint64(29)
    h *= np.uint64(0x94D049BB133111EB)
    h ^= h >> np.uint64(32)
    return (h & np.uint64(0xFFFFFF)).astype(np.float64) / float(0xFFFFFF) * 2.0 - 1.0


def value_noise(p: np.ndarray, seed: int, octaves=4, lacunarity=2.0, gain=0.5, freq=2.0) -> np.ndarray:
    """Fractal value noise: trilinear (smoothstep) interpolation of hashed
    lattice values, ``octaves`` octaves. Returns values roughly in [-1, 1]."""
    total = np.zeros(p.shape[0])
    amp, norm = 1.0, 0.0
    with np.errstate(over="ignore"):
        for o in range(octaves):
            q = p * freq
            i0 = np.floor(q).astype(np.int64)
            f = q - i0
            w = f * f * (3.0 - 2.0 * f)
            acc = np.zeros(p.shape[0])
            for dx in (0, 1):
                for dy in (0, 1):
                    for dz in (0, 1):
                        v = _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed * 131 + o)
                        wx = w[:, 0] if dx else 1 - w[:, 0]
                        wy = w[:, 1] if dy else 1 - w[:, 1]
                        wz = w[:, 2] if dz else 1 - w[:, 2]
                        acc += v * wx * wy * wz
            total += amp * acc
            norm += amp
            amp *= gain
            freq *= lacunarity
    return total / norm


def icosphere(level: int):
    """Unit icosphere subdivided ``level`` times: 20 * 4**level faces."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(level):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b2 = uniq // (nv + 1), uniq % (nv + 1)
        mid = v[a] + v[b2]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + nv  # midpoints of edges (01, 12, 20)
        f = np.concatenate([np.stack([f[:, 0], m[:, 0], m[:, 2]], 1), np.stack([f[:, 1], m[:, 1], m[:, 0]], 1),
                            np.stack([f[:, 2], m[:, 2], m[:, 1]], 1), m])
    return v, f


def torus_knot(n_u: int, n_v: int, p=2, q=3, R=0.5, r_tube=0.12):
    """(p,q) torus knot swept with a circular tube: ``2 * n_u * n_v`` faces.
    Returns unit-free vertices, faces and the per-vertex outward tube normal."""
    u = np.arange(n_u) / n_u * 2 * np.pi
    def curve(t):
        rr = R * (2 + np.cos(q * t)) / 3.0
        return np.stack([rr * np.cos(p * t), R * np.sin(q * t) / 3.0 * 1.0, rr * np.sin(p * t)], 1)
    c = curve(u)
    dc = curve(u + 1e-4) - curve(u - 1e-4)
    tng = dc / np.linalg.norm(dc, axis=1, keepdims=True)
    ref = np.array([0.0, 1.0, 0.0])
    nrm = np.cross(tng, ref)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    bin_ = np.cross(tng, nrm)
    vv = np.arange(n_v) / n_v * 2 * np.pi
    dirs = (np.cos(vv)[None, :, None] * nrm[:, None, :] + np.sin(vv)[None, :, None] * bin_[:, None, :])
    verts = (c[:, None, :] + r_tube * dirs).reshape(-1, 3)
    iu, iv = np.meshgrid(np.arange(n_u), np.arange(n_v), indexing="ij")
    a = iu * n_v + iv
    b2 = ((iu + 1) % n_u) * n_v + iv
    c2 = ((iu + 1) % n_u) * n_v + (iv + 1) % n_v
    d = iu * n_v + (iv + 1) % n_v
    faces = np.concatenate([np.stack([a, b2, c2], -1).reshape(-1, 3), np.stack([a, c2, d], -1).reshape(-1, 3)])
    return verts, faces, dirs.reshape(-1, 3)


def vertex_normals(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    """Area-weighted smooth normals of a triangle mesh."""
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)


def displaced_icosphere(level: int, radius: float, center, seed: int, amplitude=0.05):
    v, f = icosphere(level)
    d = value_noise(v * 1.0, seed)
    v = v * (radius * (1.0 + amplitude * d))[:, None] + np.asarray(center, np.float64)
    v32 = v.astype(np.float32)
    n = vertex_normals(v32.astype(np.float64), f)
    return v32, n.astype(np.float32), f


def procedural_mesh_box(level=8, res=1024, spp=64, max_depth=16, rr_depth=5, seed_mesh=2, seed_alpha=3,
                        groups=64) -> SceneDesc:
    """Noise-displaced icosphere (20 * 4**level faces; level 8 = 1,310,720) of
    radius 0.4 at (0, -0.55, 0) in the Cornell box (no spheres), GGX conductor
    with eta = k = 1.5 (as Gyunity_exe/CornellBox.h:417-422) and alpha ~
    U(0.05, 0.5) per contiguous face group."""
    b = _Builder()
    _cornell_walls(b)
    v, n, f = displaced_icosphere(level, 0.4, (0.0, -0.55, 0.0), seed_mesh)
    rng = np.random.default_rng(seed_alpha)
    alphas = rng.uniform(0.05, 0.5, groups)
    mats = [b.material(*_mat(MAT_CONDUCTOR, (1, 1, 1), ax=a, ay=a)) for a in alphas]
    per = max(1, f.shape[0] // groups)
    grp = np.minimum(np.arange(f.shape[0]) // per, groups - 1)
    b.tris(v, n, f, np.asarray(mats, np.uint32)[grp])
    return b.build(camera=Camera(res_x=res, res_y=res), params=RenderParams(spp, max_depth, rr_depth),
                   name="icosphere_L%d_%dx%d_%dspp" % (level, res, res, spp))


def mixed_materials_box(level=3, res=64, spp=4, max_depth=8, rr_depth=3, seed=11) -> SceneDesc:
    """Small test scene touching every material kind: Cornell walls and light,
    a displaced icosphere split into diffuse / conductor / rough-dielectric
    thirds, and a mirror and a glass sphere."""
    b = _Builder()
    _cornell_walls(b)
    v, n, f = displaced_icosphere(level, 0.35, (0.0, -0.3, 0.0), seed)
    diff = b.material(*_mat(MAT_DIFFUSE, (0.6, 0.7, 0.5)))
    cond = b.material(*_mat(MAT_CONDUCTOR, (0.9, 0.8, 0.7), ax=0.2, ay=0.2))
    diel = b.material(*_mat(MAT_DIELECTRIC, (1, 1, 1), (1, 1, 1), ax=0.1, ay=0.1, eta=1.5))
    third = f.shape[0] // 3
    mats = np.where(np.arange(f.shape[0]) < third, diff, np.where(np.arange(f.shape[0]) < 2 * third, cond, diel))
    b.tris(v, n, f, mats)
    mirror = b.material(*_mat(MAT_MIRROR, (1, 1, 1)))
    glass = b.material(*_mat(MAT_GLASS, (1, 1, 1), (1, 1, 1), eta=1.5, eta1=1.0))
    return b.build(camera=Camera(res_x=res, res_y=res), params=RenderParams(spp, max_depth, rr_depth),
                   spheres=np.array([[-0.55, -0.7, -0.4, 0.25], [0.55, -0.7, 0.4, 0.25]], np.float32),
                   sphere_material=np.array([mirror, glass], np.uint32), name="mixed_materials_box")


# ------------------------------------------------ differentiable rendering ---

@dataclasses.dataclass
class InverseParams:
    """The optimised parameters of inverse_box: per material group albedo
    (g, 3) and GGX alpha (g,), per emitter radiance (e, 3)."""
    albedo: np.ndarray
    alpha: np.ndarray
    radiance: np.ndarray

    def flat(self) -> np.ndarray:
        return np.concatenate([self.albedo.ravel(), self.alpha.ravel(), self.radiance.ravel()]).astype(np.float64)

    @property
    def count(self) -> int:
        return self.albedo.size + self.alpha.size + self.radiance.size


def inverse_params(groups=256, emitters=4, seed=7) -> InverseParams:
    """Hidden parameters (seeded): albedo ~ U(0.2, 0.9) per channel, alpha ~
    U(0.05, 0.5), emitter radiance 4 * U(0.75, 1.25) per channel."""
    rng = np.random.default_rng(seed)
    return InverseParams(rng.uniform(0.2, 0.9, (groups, 3)), rng.uniform(0.05, 0.5, groups),
                         4.0 * rng.uniform(0.75, 1.25, (emitters, 3)))


def perturb_params(p: InverseParams, seed=8, spread=0.3) -> InverseParams:
    """Initial parameters: every value times U(1 - spread, 1 + spread)."""
    rng = np.random.default_rng(seed)
    return InverseParams(p.albedo * rng.uniform(1 - spread, 1 + spread, p.albedo.shape),
                         p.alpha * rng.uniform(1 - spread, 1 + spread, p.alpha.shape),
                         p.radiance * rng.uniform(1 - spread, 1 + spread, p.radiance.shape))


def inverse_box(params: InverseParams = None, level=5, res=512, spp=32, max_depth=8, rr_depth=8,
                emitter_half=0.15) -> SceneDesc:
    """Inverse-rendering scene: the Cornell walls (no central light), a level-
    ``level`` icosphere (20 * 4**level faces; level 5 = 20,480) of radius 0.45
    at (0, -0.4, 0) split into len(params.alpha) contiguous face groups, each a
    GGX conductor (eta = k = 1.5) with its own albedo and alpha, and one
    emitter quad per radiance row near each ceiling corner (both triangles of
    a quad share one emission row). Roulette starts at rr_depth (>= max_depth:
    none), so the estimator is smooth in the parameters."""
    params = params or inverse_params()
    groups = params.alpha.shape[0]
    b = _Builder()
    _cornell_walls(b, light=False)
    v, n, f = displaced_icosphere(level, 0.45, (0.0, -0.4, 0.0), 5, amplitude=0.03)
    first = len(b.mt)
    for g in range(groups):
        a = float(params.alpha[g])
        b.material(*_mat(MAT_CONDUCTOR, tuple(float(x) for x in params.albedo[g]), ax=a, ay=a))
    per = f.shape[0] // groups
    grp = np.minimum(np.arange(f.shape[0]) // per, groups - 1)
    b.tris(v, n, f, (first + grp).astype(np.uint32))
    black = b.material(*_mat(MAT_DIFFUSE, (0.0, 0.0, 0.0)))
    h = emitter_half
    y = 0.965
    corners = [(-0.6, -0.6), (0.6, -0.6), (0.6, 0.6), (-0.6, 0.6)]
    for k, (cx, cz) in enumerate(corners[:params.radiance.shape[0]]):
        q = [(cx + h, y, cz + h), (cx + h, y, cz - h), (cx - h, y, cz - h), (cx - h, y, cz + h)]
        base = b.nv
        b.v.append(np.array(q, np.float32))
        b.n.append(np.array([(0, -1, 0)] * 4, np.float32))
        b.nv += 4
        b.i.append(np.array([[base, base + 1, base + 2], [base, base + 2, base + 3]], np.uint32))
        b.tm += [black, black]
        row = len(b.em)
        b.em.append(tuple(float(x) for x in params.radiance[k]))
        b.te += [row, row]
    sd = b.build(camera=Camera(res_x=res, res_y=res), params=RenderParams(spp, max_depth, rr_depth),
                 name="inverse_box_L%d_%dgroups_%dx%d_%dspp" % (level, groups, res, res, spp))
    sd.param_materials = np.arange(first, first + groups, dtype=np.int64)
    return sd


def apply_inverse_params(sd: SceneDesc, p: InverseParams):
    """Material parameters (n_materials, 16) and emission (n_emission, 3) of
    inverse_box's scene with the given optimised parameters."""
    mp = sd.mat_params.copy()
    m = sd.param_materials
    mp[m, 0:3] = p.albedo
    mp[m, 6] = p.alpha
    mp[m, 7] = p.alpha
    em = p.radiance.astype(np.float32).copy()
    return np.ascontiguousarray(mp, np.float32), np.ascontiguousarray(em, np.float32)


# ------------------------------------------------- batched uneven workload ---

def _smooth_normals(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals with one bincount per axis (the batch
    workload's meshes; vertex_normals keeps the older summation order for the
    scenes the golden fixtures were made from)."""
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    idx = f.reshape(-1)
    n = np.stack([np.bincount(idx, np.repeat(fn[:, a], 3), minlength=v.shape[0]) for a in range(3)], 1)
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)


_ICO_CACHE = {}


def _unit_icosphere(level: int):
    if level not in _ICO_CACHE:
        _ICO_CACHE[level] = icosphere(level)
    v, f = _ICO_CACHE[level]
    return v.copy(), f


def ring_torus(n_u: int, n_v: int, R=0.42, r=0.16):
    """Ring torus around the y axis: 2 * n_u * n_v faces; returns vertices,
    faces and the outward tube direction per vertex."""
    u = np.arange(n_u) / n_u * 2 * np.pi
    w = np.arange(n_v) / n_v * 2 * np.pi
    cu, su, cw, sw = np.cos(u)[:, None], np.sin(u)[:, None], np.cos(w)[None, :], np.sin(w)[None, :]
    dirs = np.stack([cu * cw, np.broadcast_to(sw, (n_u, n_v)), su * cw], -1).reshape(-1, 3)
    center = np.stack([R * cu[:, 0], np.zeros(n_u), R * su[:, 0]], 1)
    verts = (np.repeat(center, n_v, 0) + r * dirs)
    iu, iv = np.meshgrid(np.arange(n_u), np.arange(n_v), indexing="ij")
    a = iu * n_v + iv
    b2 = ((iu + 1) % n_u) * n_v + iv
    c2 = ((iu + 1) % n_u) * n_v + (iv + 1) % n_v
    d = iu * n_v + (iv + 1) % n_v
    faces = np.concatenate([np.stack([a, c2, b2], -1).reshape(-1, 3), np.stack([a, d, c2], -1).reshape(-1, 3)])
    return verts, faces, dirs


def batch_instance(seed: int, min_tris=10_000, max_tris=2_000_000, max_depth=16, rr_depth=5) -> SceneDesc:
    """One instance of the uneven batch workload (seeded): a Cornell box
    (walls and ceiling light as cornell_box, no spheres) holding a noise-
    displaced icosphere or ring torus (coin flip) of log-uniform triangle count
    in [min_tris, max_tris] (icospheres: the nearest subdivision level, tori:
    a grid of about that many faces), diffuse or GGX-conductor (coin flip)
    with albedo ~ U(0.2, 0.9) per channel and alpha ~ U(0.05, 0.5);
    resolution uniform in {128, 256, 512, 1024} squared, spp uniform in 1..64."""
    rng = np.random.default_rng(seed)
    target = float(np.exp(rng.uniform(np.log(min_tris), np.log(max_tris))))
    torus = bool(rng.integers(0, 2))
    diffuse = bool(rng.integers(0, 2))
    albedo = tuple(float(a) for a in rng.uniform(0.2, 0.9, 3))
    alpha = float(rng.uniform(0.05, 0.5))
    res = int(rng.choice([128, 256, 512, 1024]))
    spp = int(rng.integers(1, 65))
    b = _Builder()
    _cornell_walls(b)
    if torus:
        n_u = max(8, int(round(math.sqrt(target))))
        n_v = max(4, int(round(target / (2 * n_u))))
        v, f, dirs = ring_torus(n_u, n_v)
        d = value_noise(v, seed)
        v = v + dirs * (0.16 * 0.05 * d)[:, None] + np.array([0.0, -0.55, 0.0])
    else:
        level = int(np.clip(round(math.log(target / 20.0, 4)), 2, 8))
        v, f = _unit_icosphere(level)
        d = value_noise(v, seed)
        v = v * (0.42 * (1.0 + 0.05 * d))[:, None] + np.array([0.0, -0.5, 0.0])
    v32 = v.astype(np.float32)
    n = _smooth_normals(v32.astype(np.float64), f).astype(np.float32)
    if diffuse:
        m = b.material(*_mat(MAT_DIFFUSE, albedo))
    else:
        m = b.material(*_mat(MAT_CONDUCTOR, albedo, ax=alpha, ay=alpha))
    b.tris(v32, n, f, np.full(f.shape[0], m, np.uint32))
    return b.build(camera=Camera(res_x=res, res_y=res), params=RenderParams(spp, max_depth, rr_depth),
                   name="batch_%d_%s_%d_%dx%d_%dspp" % (seed, "torus" if torus else "ico", f.shape[0], res, res, spp))


def batch_workload(n=64, seed=1000, **kw):
    """The uneven batch: instances seed, seed + 1, ..., seed + n - 1."""
    return [batch_instance(seed + i, **kw) for i in range(n)]


# ----------------------------------------------------------- environment ---

def rgbe_quantize(img: np.ndarray) -> np.ndarray:
    """Round an RGB float image to the values an RGBE (.hdr) file stores:
    shared exponent from frexp of the largest component, 8-bit mantissas by
    truncation, decoded as mantissa * 2^(exponent - 8) (Ward's RGBE format).
    The result survives a write/read round trip unchanged, so an environment
    map given to the reference through a file and to the GPU directly holds
    identical texels."""
    img = np.ascontiguousarray(img, np.float32)
    m = img.max(axis=2)
    mant, ex = np.frexp(m.astype(np.float64))
    with np.errstate(divide="ignore", invalid="ignore"):
        normalize = (mant.astype(np.float32) * np.float32(256.0)) / m
        b = np.trunc(img * normalize[..., None]).astype(np.int64) % 256
    out = (b.astype(np.float64) * np.ldexp(1.0, (ex - 8))[..., None]).astype(np.float32)
    out[m < np.float32(1e-32)] = 0.0
    return out


def sky_envmap(width=2048, height=1024, seed=5, sun_elevation_deg=45.0, sun_azimuth_deg=30.0,
               sun_diameter_deg=0.5, sun_radiance=None):
    """Synthetic lat-long sky: zenith (0.3, 0.5, 1.0) to horizon 0.8 gradient
    above the horizon, ground 0.1 below, plus a sun disk whose radiance is one
    draw from lognormal(mu=8, sigma=1). Row 0 is the zenith (theta = 0) and
    directions follow EnvironmentMap::LatLongToDir (light/EnvMap.h:92-100):
    (sin(theta) cos(phi), cos(theta), sin(theta) sin(phi))."""
    rng = np.random.default_rng(seed)
    if sun_radiance is None:
        sun_radiance = float(rng.lognormal(8.0, 1.0))
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = v[:, None] * np.pi
    phi = u[None, :] * 2 * np.pi
    d = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta) * np.ones_like(phi), np.sin(theta) * np.sin(phi)], -1)
    y = d[..., 1:2]
    zen = np.array([0.3, 0.5, 1.0])
    hor = np.array([0.8, 0.8, 0.8])
    t = np.clip(y, 0, 1)
    img = np.where(y > 0, hor * (1 - t) + zen * t, 0.1)
    el, az = np.radians(sun_elevation_deg), np.radians(sun_azimuth_deg)
    sdir = np.array([np.cos(el) * np.cos(az), np.sin(el), np.cos(el) * np.sin(az)])
    cosang = (d * sdir).sum(-1)
    disk = cosang >= np.cos(np.radians(sun_diameter_deg / 2))
    img[disk] = sun_radiance
    return rgbe_quantize(img.astype(np.float32))


def env_torus_knot(n_u=2000, n_v=1000, res_x=1920, res_y=1080, spp=256, max_depth=32, rr_depth=5, seed=4,
                   env_w=2048, env_h=1024, sun_diameter_deg=0.5, alpha=0.1) -> SceneDesc:
    """Environment-lit rough glass: a (2,3) torus knot tube swept with
    n_u x n_v quads (2 n_u n_v triangles; 2000 x 1000 = 4M), displaced by 5% of
    the tube radius with 4-octave value noise, GGX rough dielectric
    (alpha 0.1, IOR 1.5), lit only by the synthetic sky map."""
    b = _Builder()
    v, f, nrm = torus_knot(n_u, n_v)
    r_tube = 0.12
    disp = value_noise(v * 2.0, seed)
    v = v + nrm * (0.05 * r_tube * disp)[:, None]
    v32 = v.astype(np.float32)
    n = vertex_normals(v32.astype(np.float64), f)
    glass = b.material(*_mat(MAT_DIELECTRIC, (1, 1, 1), (1, 1, 1), ax=alpha, ay=alpha, eta=1.5))
    b.tris(v32, n.astype(np.float32), f, np.full(f.shape[0], glass, np.uint32))
    env = sky_envmap(env_w, env_h, seed=5, sun_diameter_deg=sun_diameter_deg)
    return b.build(camera=Camera(res_x=res_x, res_y=res_y), params=RenderParams(spp, max_depth, rr_depth),
                   env=env, env_scale=1.0, name="env_torus_knot_%dtris" % f.shape[0])


def env_knot_small() -> SceneDesc:
    """Small environment-lit rough-glass scene for tests: 3,840 triangles,
    128 x 64 sky map with a 12-degree sun, 96 x 54 film, 4 spp, depth 8."""
    return env_torus_knot(n_u=120, n_v=16, res_x=96, res_y=54, spp=4, max_depth=8, env_w=128, env_h=64,
                          sun_diameter_deg=12)
