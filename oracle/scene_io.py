"""Binary I/O between the tests and the reference harness (oracle/ref/harness.cpp).

TEST INFRASTRUCTURE ONLY: only tests/, the golden-vector generator and
bench.py's CPU-baseline leg use this module.

Scene file (little-endian), read by ``load_scene`` in the harness:
  u32 magic 'GYTS', u32 version=1,
  u32 nv, nt, ns, nm, ne, has_normals, env_w, env_h,
  u32 res_x, res_y, spp, max_depth, rr_depth,
  f32 camera[11] = pos[3], look_at[3], up[3], fovy, film_distance,
  f32 env_scale,
  f32 vertices[nv*3], [f32 normals[nv*3] if has_normals], u32 indices[nt*3],
  u32 tri_material[nt], i32 tri_emission[nt], f32 spheres[ns*4],
  u32 sphere_material[ns], u32 mat_type[nm], f32 mat_params[nm*16],
  f32 emission[ne*3], f32 env[env_h*env_w*3] (row 0 = top).
"""
import os
import subprocess
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "gyref_harness")


def write_scene(path, sd):
    ns = sd.n_spheres
    env = sd.env
    env_h, env_w = (0, 0) if env is None else env.shape[:2]
    c = sd.camera
    p = sd.params
    media = getattr(sd, "media", None)
    tri_medium = getattr(sd, "tri_medium", None)
    version = 2 if media is not None else 1
    with open(path, "wb") as f:
        f.write(struct.pack("<2I", 0x53545947, version))
        f.write(struct.pack("<8I", sd.vertices.shape[0], sd.n_triangles, ns, sd.mat_type.shape[0],
                            sd.emission.shape[0], 0 if sd.normals is None else 1, env_w, env_h))
        f.write(struct.pack("<5I", c.res_x, c.res_y, p.spp, p.max_depth, p.rr_depth))
        f.write(np.array(list(c.pos) + list(c.look_at) + list(c.up) + [c.fovy, c.film_distance], np.float32).tobytes())
        f.write(struct.pack("<f", sd.env_scale))
        f.write(np.ascontiguousarray(sd.vertices, np.float32).tobytes())
        if sd.normals is not None:
            f.write(np.ascontiguousarray(sd.normals, np.float32).tobytes())
        f.write(np.ascontiguousarray(sd.indices, np.uint32).tobytes())
        f.write(np.ascontiguousarray(sd.tri_material, np.uint32).tobytes())
        f.write(np.ascontiguousarray(sd.tri_emission, np.int32).tobytes())
        if ns:
            f.write(np.ascontiguousarray(sd.spheres, np.float32).tobytes())
            f.write(np.ascontiguousarray(sd.sphere_material, np.uint32).tobytes())
        f.write(np.ascontiguousarray(sd.mat_type, np.uint32).tobytes())
        f.write(np.ascontiguousarray(sd.mat_params, np.float32).tobytes())
        f.write(np.ascontiguousarray(sd.emission, np.float32).tobytes())
        if env is not None:
            f.write(np.ascontiguousarray(env, np.float32).tobytes())
        if version == 2:
            # version 2: homogeneous media and per-triangle medium interfaces
            m = np.ascontiguousarray(media, np.float32).reshape(-1, 7)
            f.write(struct.pack("<2I", m.shape[0], 0 if tri_medium is None else 1))
            f.write(m.tobytes())
            if tri_medium is not None:
                f.write(np.ascontiguousarray(tri_medium, np.int32).reshape(-1, 2).tobytes())


def have_harness():
    return os.path.exists(HARNESS)


def run(*args, env=None):
    e = dict(os.environ)
    if env:
        e.update(env)
    r = subprocess.run([HARNESS] + [str(a) for a in args], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                       text=True, env=e)
    if r.returncode != 0:
        raise RuntimeError("gyref_harness %s failed: %s" % (args[0], r.stderr[-2000:]))
    return r.stdout


RAY_DTYPE = np.dtype([("o", "<f4", 3), ("d", "<f4", 3), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("prim", "<i4"), ("t", "<f4"), ("b1", "<f4"), ("b2", "<f4")])


def ref_sobol(tmp, dims, indices):
    pairs = np.zeros(len(dims), np.dtype([("d", "<u4"), ("i", "<u8")]))
    pairs["d"] = dims
    pairs["i"] = indices
    a, b = os.path.join(tmp, "sobol_in.bin"), os.path.join(tmp, "sobol_out.bin")
    pairs.tofile(a)
    run("sobol", a, b)
    return np.fromfile(b, np.float32)


def ref_enum(tmp, res_x, res_y, s, x, y):
    trip = np.stack([np.asarray(s, np.uint32), np.asarray(x, np.uint32), np.asarray(y, np.uint32)], 1)
    a, b = os.path.join(tmp, "enum_in.bin"), os.path.join(tmp, "enum_out.bin")
    trip.astype(np.uint32).tofile(a)
    run("enum", res_x, res_y, a, b)
    return np.fromfile(b, np.uint64)


def ref_halton(tmp, dims, indices):
    """HaltonSampler with Faure permutations (sampler/Halton.h) for (dim, index) pairs."""
    pairs = np.zeros(len(dims), np.dtype([("d", "<u4"), ("i", "<u8")]))
    pairs["d"] = dims
    pairs["i"] = indices
    a, b = os.path.join(tmp, "halton_in.bin"), os.path.join(tmp, "halton_out.bin")
    pairs.tofile(a)
    run("halton", a, b)
    return np.fromfile(b, np.float32)


def ref_henum(tmp, res_x, res_y, s, x, y):
    """HaltonEnum::GetIndex (sampler/HaltonEnum.h) for (s, x, y) triplets."""
    trip = np.stack([np.asarray(s, np.uint32), np.asarray(x, np.uint32), np.asarray(y, np.uint32)], 1)
    a, b = os.path.join(tmp, "henum_in.bin"), os.path.join(tmp, "henum_out.bin")
    trip.astype(np.uint32).tofile(a)
    run("henum", res_x, res_y, a, b)
    return np.fromfile(b, np.uint64)


def _sampler_env(sampler, integrator=None):
    env = {}
    if sampler and sampler != "sobol":
        env["GYREF_SAMPLER"] = sampler
    if integrator and integrator != "pt":
        env["GYREF_INTEGRATOR"] = integrator
    return env or None


def ref_hits(tmp, scene_path, rays, any_hit=False):
    a, b = os.path.join(tmp, "rays.bin"), os.path.join(tmp, "hits.bin")
    rays.astype(RAY_DTYPE).tofile(a)
    run("anyhit" if any_hit else "hits", scene_path, a, b)
    return np.fromfile(b, HIT_DTYPE)


def ref_paths(tmp, scene_path, x, y, s, sampler=None, integrator=None):
    """Li of PathTracing (or VolPathTracing with integrator="vpt") for (x, y, s)."""
    trip = np.stack([np.asarray(x, np.uint32), np.asarray(y, np.uint32), np.asarray(s, np.uint32)], 1)
    a, b = os.path.join(tmp, "paths_in.bin"), os.path.join(tmp, "paths_out.bin")
    trip.astype(np.uint32).tofile(a)
    run("paths", scene_path, a, b, env=_sampler_env(sampler, integrator))
    return np.fromfile(b, np.float32).reshape(-1, 4)


def ref_sample(tmp, items, warmup, steps, sampler=None, threads=None):
    """PathTracing::Li of the reference over many scenes, timed: items is a
    list of (scene path, (n, 3) uint32 x, y, s samples); each scene is loaded
    (untimed) and its samples traced warmup + steps times on the host threads.
    Returns the harness's record: paths_per_step, step_s (seconds of each
    step summed over the scenes), load_s, threads."""
    import json
    lst = os.path.join(tmp, "sample_list.txt")
    with open(lst, "w") as f:
        for k, (scene_path, xys) in enumerate(items):
            trip = os.path.join(tmp, "sample_%d.bin" % k)
            np.ascontiguousarray(xys, np.uint32).tofile(trip)
            f.write("%s %s\n" % (scene_path, trip))
    env = dict(_sampler_env(sampler) or {})
    if threads:
        env["GYREF_THREADS"] = str(threads)
    out = run("sample", lst, int(warmup), int(steps), env=env or None)
    return json.loads(out.strip().splitlines()[-1])


def ref_camera(tmp, scene_path):
    b = os.path.join(tmp, "camera.bin")
    run("camera", scene_path, b)
    return np.fromfile(b, np.float32).reshape(4, 4)


def ref_render(tmp, scene_path, rows=None, spp=None, threads=None, sampler=None, integrator=None):
    import json
    b = os.path.join(tmp, "render.bin")
    args = ["render", scene_path, b]
    if rows is not None or spp is not None:
        args.append(rows if rows is not None else 0)
    if spp is not None:
        args.append(spp)
    env = dict(_sampler_env(sampler, integrator) or {})
    if threads:
        env["GYREF_THREADS"] = str(threads)
    out = run(*args, env=env or None)
    info = json.loads(out.strip().splitlines()[-1])
    img = np.fromfile(b, np.float32).reshape(-1, 4)
    return img, info


def ref_toint(tmp, x, gamma):
    """ImageIO::toInt (image/ImageIO.cpp:66-68) of float values."""
    a, b = os.path.join(tmp, "toint_in.bin"), os.path.join(tmp, "toint_out.bin")
    np.ascontiguousarray(x, np.float32).tofile(a)
    run("toint", a, repr(float(gamma)), b)
    return np.fromfile(b, np.int32)


def ref_write_image(tmp, rgb, path):
    """ImageIO::WriteImage (image/ImageIO.cpp:117-149) of a float RGB image
    (h, w, 3) to path (.png, .bmp or .hdr)."""
    a = os.path.join(tmp, "image_in.bin")
    rgb = np.ascontiguousarray(rgb, np.float32)
    rgb.tofile(a)
    run("image", a, rgb.shape[1], rgb.shape[0], path)


def ref_light_paths(tmp, scene_path, photons, sampler=None):
    """LightTracing per photon: (n, max_depth, 6) records (on film 1/0 or -1,
    X, Y, splatted RGB)."""
    a, b = os.path.join(tmp, "lt_in.bin"), os.path.join(tmp, "lt_out.bin")
    np.ascontiguousarray(photons, np.uint64).tofile(a)
    run("lt", scene_path, a, b, env=_sampler_env(sampler))
    return np.fromfile(b, np.float32).reshape(len(photons), -1, 6)


def ref_light_render(tmp, scene_path, sampler=None):
    """LightTracing::Render: the film's splat buffer (h, w, 3) and the timing."""
    import json
    b = os.path.join(tmp, "ltimg.bin")
    out = run("ltrender", scene_path, b, env=_sampler_env(sampler))
    info = json.loads(out.strip().splitlines()[-1])
    return np.fromfile(b, np.float32), info


def ref_obj(tmp, obj_path, reverse, spec):
    """Mesh::LoadFromFile of obj_path, then Triangle::SetTransform by the
    transform spec ("-" for none): (n, 6, 3) float32 p0 p1 p2 n0 n1 n2."""
    b = os.path.join(tmp, "obj_out.bin")
    run("obj", obj_path, int(reverse), spec, b)
    return np.fromfile(b, np.float32).reshape(-1, 6, 3)


def ref_bsdf(tmp, cases):
    """cases: structured array with fields type (u4), params (16 f4), wo, u, we (3 f4)."""
    a, b = os.path.join(tmp, "bsdf_in.bin"), os.path.join(tmp, "bsdf_out.bin")
    cases.tofile(a)
    run("bsdf", a, b)
    return np.fromfile(b, np.float32).reshape(-1, 11)


BSDF_CASE_DTYPE = np.dtype([("type", "<u4"), ("params", "<f4", 16), ("wo", "<f4", 3), ("u", "<f4", 3),
                            ("we", "<f4", 3)])
