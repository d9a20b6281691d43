"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference renderer compiled from its own sources by
oracle/ref/build_ref.py (``oracle/_ref/gyref_harness``) on seeded inputs and
stores the inputs and the reference outputs as .npz fixtures. The reference
checkout is only needed to regenerate; the tests read the fixtures.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py halton     # only the Halton fixtures
    python tests/golden/make_golden.py film       # only the film-output fixtures
    python tests/golden/make_golden.py obj        # only the OBJ-mesh fixtures
    python tests/golden/make_golden.py lt         # only the light-tracing fixtures
    python tests/golden/make_golden.py vpt        # only the volume fixtures
    python tests/golden/make_golden.py vpt_eq     # only the equi-angular volume fixtures
    python tests/golden/make_golden.py zstat      # only the per-pixel moments of the z-test
"""
import dataclasses
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gyunity_b200 import scenes  # noqa: E402
from oracle import scene_io as io  # noqa: E402


def random_rays(sd, n, rng):
    """Rays from inside the box towards random directions, plus camera-like
    rays through the open front, with finite and infinite tmax."""
    o = rng.uniform(-0.95, 0.95, (n, 3)).astype(np.float32)
    half = n // 2
    o[half:, 2] = 2.9
    d = rng.normal(size=(n, 3))
    d[half:, 2] = -np.abs(d[half:, 2]) - 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.2, rng.uniform(0.1, 2.0, n), np.inf).astype(np.float32)
    rays = np.zeros(n, io.RAY_DTYPE)
    rays["o"] = o
    rays["d"] = d.astype(np.float32)
    rays["tmax"] = tmax
    return rays


def bsdf_cases(rng, n_per=400):
    cases = []
    kinds = [
        (0, dict(a=(0.7, 0.5, 0.3))),
        (1, dict(a=(0.9, 0.9, 0.9))),
        (2, dict(a=(1, 1, 1), b=(1, 1, 1), eta=1.5, eta1=1.0)),
        (3, dict(a=(1, 1, 1), ax=0.05, ay=0.05)), (3, dict(a=(1, 1, 1), ax=0.2, ay=0.2)),
        (3, dict(a=(0.9, 0.8, 0.7), ax=0.5, ay=0.5)),
        (4, dict(a=(1, 1, 1), b=(1, 1, 1), ax=0.1, ay=0.1, eta=1.5)),
        (4, dict(a=(1, 1, 1), b=(1, 1, 1), ax=0.5, ay=0.5, eta=1.5)),
    ]
    for kind, kw in kinds:
        _, p = scenes._mat(kind, **kw)
        c = np.zeros(n_per, io.BSDF_CASE_DTYPE)
        c["type"] = kind
        c["params"] = p
        wo = rng.normal(size=(n_per, 3))
        wo /= np.linalg.norm(wo, axis=1, keepdims=True)
        we = rng.normal(size=(n_per, 3))
        we /= np.linalg.norm(we, axis=1, keepdims=True)
        c["wo"] = wo.astype(np.float32)
        c["u"] = rng.uniform(size=(n_per, 3)).astype(np.float32)
        c["we"] = we.astype(np.float32)
        cases.append(c)
    return np.concatenate(cases)


def halton_golden(tmp):
    """HaltonSampler (Faure permutations), HaltonEnum and PathTracing::Li with
    the Halton sampler (GYREF_SAMPLER=halton selects it in the harness)."""
    rng = np.random.default_rng(20261204)
    # all 256 dimensions (and some beyond, which give 0) at small, 32-bit and 44-bit indices
    dims = np.concatenate([np.arange(300), np.arange(300), rng.integers(0, 256, 3000)]).astype(np.uint32)
    idx = np.concatenate([rng.integers(0, 1 << 20, 300), rng.integers(0, 1 << 44, 300),
                          rng.integers(0, 1 << 32, 1500), rng.integers(0, 1 << 44, 1500)]).astype(np.uint64)
    np.savez_compressed(os.path.join(HERE, "halton.npz"), dims=dims, indices=idx,
                        values=io.ref_halton(tmp, dims, idx))
    enum = {}
    for rx, ry in ((256, 256), (1024, 1024), (1920, 1080), (100, 60), (1, 1), (7, 1), (1, 5)):
        s = rng.integers(0, 300, 800).astype(np.uint32)
        x = rng.integers(0, rx, 800).astype(np.uint32)
        y = rng.integers(0, ry, 800).astype(np.uint32)
        key = "%dx%d" % (rx, ry)
        enum[key + "_sxy"] = np.stack([s, x, y], 1)
        enum[key + "_index"] = io.ref_henum(tmp, rx, ry, s, x, y)
    np.savez_compressed(os.path.join(HERE, "henum.npz"), **enum)
    for name, sd in (("cornell_nospheres", scenes.cornell_box(spheres=False)),
                     ("mixed", scenes.mixed_materials_box(level=3, res=64))):
        sd.params.sampler = "halton"
        path = os.path.join(tmp, name + "_h.gyts")
        io.write_scene(path, sd)
        n = 3000
        x = rng.integers(0, sd.camera.res_x, n)
        y = rng.integers(0, sd.camera.res_y, n)
        s = rng.integers(0, sd.params.spp, n)
        r = io.ref_paths(tmp, path, x, y, s, sampler="halton")
        np.savez_compressed(os.path.join(HERE, "paths_%s_halton.npz" % name),
                            xys=np.stack([x, y, s], 1).astype(np.uint32), L=r[:, :3], cursor=r[:, 3].astype(np.int32))
    sd = scenes.cornell_box(res=64, spp=4)
    sd.params.sampler = "halton"
    path = os.path.join(tmp, "img_h.gyts")
    io.write_scene(path, sd)
    img, info = io.ref_render(tmp, path, sampler="halton")
    np.savez_compressed(os.path.join(HERE, "image_cornell_64x64_4spp_halton.npz"), film=img)


def film_output_golden(tmp):
    """ImageIO::toInt at three gammas and ImageIO::WriteImage of one float
    image to .png, .bmp and .hdr (decoded pixels stored)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from image_tools import read_hdr_rgbe, read_rgb8
    rng = np.random.default_rng(20261205)
    x = np.concatenate([rng.uniform(-0.2, 1.3, 15000), np.linspace(0.0, 1.0, 5001),
                        np.array([0.0, 1.0, -0.0, 1e-30, 1e-7, 0.5, 2.0, -1.0])]).astype(np.float32)
    out = {"x": x}
    for g in (2.2, 1.8, 1.0):
        out["toint_%g" % g] = io.ref_toint(tmp, x, g)
    h, w = 23, 37  # odd sizes: BMP row padding, HDR run-length scanlines
    img = np.zeros((h, w, 3), np.float32)
    img[..., 0] = np.linspace(0, 1.2, w)[None, :]
    img[..., 1] = np.linspace(-0.1, 1.0, h)[:, None]
    img[..., 2] = rng.lognormal(-1.0, 1.5, (h, w))
    img[0, 0] = 0.0
    img[1, 1] = (5000.0, 0.25, 1e-3)
    out["image"] = img
    for ext in ("png", "bmp", "hdr"):
        path = os.path.join(tmp, "ref." + ext)
        io.ref_write_image(tmp, img, path)
        out["decoded_" + ext] = read_hdr_rgbe(path) if ext == "hdr" else read_rgb8(path)
    np.savez_compressed(os.path.join(HERE, "film_output.npz"), **out)


OBJ_TRANSFORMS = ["T 0 -0.5 0;S 0.28 0.28 0.28",                       # CornellBox.h:534
                  "T 0 -0.35 0;S 0.02 0.02 0.02;T -50 0 50;RX -90;S 1 2 1",  # CornellBox.h:1200-1208
                  "RY 30;RZ 45;T 0.1 0.2 0.3;S 2 3 0.5;RX 17.5"]


def obj_files(rng):
    """Synthetic OBJ files for the loader: polygons (convex, concave,
    collinear), every face-index form and number format, line endings."""
    files = {}
    # a 4x3 grid of quads with texture coordinates and normals, a pentagon, an
    # L-shaped (concave) hexagon and a quad with three collinear vertices
    lines = ["# quads and polygons", "o grid", "g grid"]
    for j in range(4):
        for i in range(5):
            z = 0.05 * np.sin(i + 2 * j)
            lines.append("v %.6f %.6f %.6f" % (i * 0.25, j * 0.3, z))
            lines.append("vt %.4f %.4f" % (i / 4, j / 3))
            lines.append("vn %.6f %.6f %.6f" % (0.1 * i, 0.05 * j, 1.0))
    for j in range(3):
        for i in range(4):
            a = 1 + i + 5 * j
            q = (a, a + 1, a + 6, a + 5)
            lines.append("f " + " ".join("%d/%d/%d" % (k, k, k) for k in q))
    lines.append("usemtl other")
    base = 20
    for ang in range(5):
        t = 2 * np.pi * ang / 5
        lines.append("v %.7f %.7f 1.5" % (np.cos(t), np.sin(t)))
    lines.append("f %s" % " ".join(str(base + 1 + k) for k in range(5)))
    lshape = [(0, 0), (2, 0), (2, 1), (1, 1), (1, 2), (0, 2)]
    for x, y in lshape:
        lines.append("v %g %g -1" % (x, y))
    lines.append("f %s" % " ".join(str(base + 6 + k) for k in range(6)))
    for x in (0, 1, 2):
        lines.append("v %d 5 0.5" % x)
    lines.append("v 1 6 0.5")
    lines.append("f -4 -3 -2 -1")
    files["polygons.obj"] = "\n".join(lines) + "\n"
    # index forms (v, v/vt, v//vn, v/vt/vn, negative), number formats, CRLF
    # line endings, tabs, comments, a face of two vertices (skipped)
    body = ["# forms", "v 1e-3 .5 -.25", "v +2 3. 1.000000001", "v -0 1E+2 0.1234567890123",
            "v\t0.5\t0.25\t-0.125  ", "vn 0 0 1", "vn 0 1 0", "vt 0.5 0.5", "vt 1 0",
            "s off", "f 1 2 3", "f 1/1 2/2 3/1", "f 1//1 2//2 4//1", "f -4/-2/-2 -3/-1/-1 -1/-2/-2",
            "f 1 2", "", "   # indented comment", "g second", "f\t2 3 4"]
    files["forms.obj"] = "\r\n".join(body) + "\r\n"
    # no normals anywhere (face normals generated), one zero-area triangle
    ico = ["v 0 0 0", "v 1 0 0", "v 0 1 0", "v 0 0 1", "v 2 0 0", "v 3 0 0",
           "f 1 2 3", "f 1 3 4", "f 1 4 2", "f 2 4 3", "f 2 5 6"]
    files["generated_normals.obj"] = "\n".join(ico) + "\n"
    # a seeded noisy sphere (latitude-longitude, quads at the poles become triangles)
    sph = []
    nu, nv = 24, 12
    for j in range(nv + 1):
        for i in range(nu):
            th, ph = np.pi * j / nv, 2 * np.pi * i / nu
            r = 1 + 0.05 * rng.standard_normal()
            sph.append("v %.7f %.7f %.7f" % (r * np.sin(th) * np.cos(ph), r * np.cos(th), r * np.sin(th) * np.sin(ph)))
    for j in range(nv):
        for i in range(nu):
            a, b = j * nu + i + 1, j * nu + (i + 1) % nu + 1
            sph.append("f %d %d %d %d" % (a, b, b + nu, a + nu))
    files["sphere.obj"] = "\n".join(sph) + "\n"
    return files


def obj_golden(tmp):
    """Mesh::LoadFromFile of the synthetic OBJ files (both vertex orders) and
    Triangle::SetTransform by three of the reference's own transforms."""
    rng = np.random.default_rng(20261206)
    odir = os.path.join(HERE, "obj")
    os.makedirs(odir, exist_ok=True)
    out = {}
    for name, text in obj_files(rng).items():
        path = os.path.join(odir, name)
        with open(path, "w", newline="") as f:
            f.write(text)
        key = name[:-4]
        for rev in (0, 1):
            out["%s_rev%d" % (key, rev)] = io.ref_obj(tmp, path, rev, "-")
        for k, spec in enumerate(OBJ_TRANSFORMS):
            out["%s_t%d" % (key, k)] = io.ref_obj(tmp, path, 0, spec)
    out["transforms"] = np.array(OBJ_TRANSFORMS)
    np.savez_compressed(os.path.join(HERE, "obj_meshes.npz"), **out)


def light_tracing_golden(tmp):
    """LightTracing per photon (records of every vertex's camera join) and
    LightTracing::Render of the Cornell box."""
    rng = np.random.default_rng(20261207)
    for name, sd in (("cornell_nospheres", scenes.cornell_box(res=64, spp=4, max_depth=6, spheres=False)),
                     ("cornell", scenes.cornell_box(res=64, spp=4, max_depth=6)),
                     ("mixed", scenes.mixed_materials_box(level=3, res=48, spp=4))):
        path = os.path.join(tmp, "lt_%s.gyts" % name)
        io.write_scene(path, sd)
        total = sd.camera.res_x * sd.camera.res_y * sd.params.spp
        ids = np.sort(rng.choice(total, 3000, replace=False)).astype(np.uint64)
        np.savez_compressed(os.path.join(HERE, "lt_paths_%s.npz" % name), photons=ids,
                            records=io.ref_light_paths(tmp, path, ids))
    sd = scenes.cornell_box(res=64, spp=16, max_depth=6)
    path = os.path.join(tmp, "lt_img.gyts")
    io.write_scene(path, sd)
    img, _ = io.ref_light_render(tmp, path)
    np.savez_compressed(os.path.join(HERE, "image_lt_cornell_64x64_16spp.npz"), splat=img.reshape(64, 64, 3))


def volume_golden(tmp):
    """VolPathTracing (without equi-angular sampling) per path and rendered,
    on the Cornell box filled with fog (scenes.cornell_fog, also with the
    Halton sampler) and on the box holding a ball of fog
    (scenes.fog_ball_box)."""
    rng = np.random.default_rng(20261208)
    halton = scenes.cornell_fog(res=48, spp=4, max_depth=6)
    halton = dataclasses.replace(halton, params=dataclasses.replace(halton.params, sampler="halton"))
    for name, sd in (("fog", scenes.cornell_fog(res=48, spp=4, max_depth=6)),
                     ("fog_thick", scenes.cornell_fog(res=48, spp=4, max_depth=6, sigma_a=0.2, sigma_s=1.5, g=-0.4,
                                                      spheres=False)),
                     ("fog_ball", scenes.fog_ball_box(res=48, spp=4, max_depth=6)),
                     ("fog_halton", halton)):
        path = os.path.join(tmp, "vpt_%s.gyts" % name)
        io.write_scene(path, sd)
        n = 3000
        x = rng.integers(0, sd.camera.res_x, n)
        y = rng.integers(0, sd.camera.res_y, n)
        s = rng.integers(0, sd.params.spp, n)
        r = io.ref_paths(tmp, path, x, y, s, sampler=sd.params.sampler, integrator="vpt")
        np.savez_compressed(os.path.join(HERE, "vpt_paths_%s.npz" % name), xys=np.stack([x, y, s], 1).astype(np.uint32),
                            L=r[:, :3], cursor=r[:, 3].astype(np.int32))
    sd = scenes.cornell_fog(res=64, spp=8, max_depth=6)
    path = os.path.join(tmp, "vpt_img.gyts")
    io.write_scene(path, sd)
    img, _ = io.ref_render(tmp, path, integrator="vpt")
    np.savez_compressed(os.path.join(HERE, "image_vpt_fog_64x64_8spp.npz"), film=img)


def volume_equi_angular_golden(tmp):
    """VolPathTracing with equi-angular sampling (its constructor's default,
    harness integrator "vpt_eq") per path on the fog scenes, and rendered on
    the Cornell box in fog."""
    rng = np.random.default_rng(20261203)
    for name, sd in (("fog", scenes.cornell_fog(res=48, spp=4, max_depth=6)),
                     ("fog_thick", scenes.cornell_fog(res=48, spp=4, max_depth=6, sigma_a=0.2, sigma_s=1.5, g=-0.4,
                                                      spheres=False)),
                     ("fog_ball", scenes.fog_ball_box(res=48, spp=4, max_depth=6))):
        path = os.path.join(tmp, "vpt_eq_%s.gyts" % name)
        io.write_scene(path, sd)
        n = 3000
        x = rng.integers(0, sd.camera.res_x, n)
        y = rng.integers(0, sd.camera.res_y, n)
        s = rng.integers(0, sd.params.spp, n)
        r = io.ref_paths(tmp, path, x, y, s, sampler=sd.params.sampler, integrator="vpt_eq")
        np.savez_compressed(os.path.join(HERE, "vpt_eq_paths_%s.npz" % name),
                            xys=np.stack([x, y, s], 1).astype(np.uint32), L=r[:, :3],
                            cursor=r[:, 3].astype(np.int32))
    sd = scenes.cornell_fog(res=64, spp=8, max_depth=6)
    path = os.path.join(tmp, "vpt_eq_img.gyts")
    io.write_scene(path, sd)
    img, _ = io.ref_render(tmp, path, integrator="vpt_eq")
    np.savez_compressed(os.path.join(HERE, "image_vpt_eq_fog_64x64_8spp.npz"), film=img)


ZSTAT_SCENES = {
    "cornell_256x256_16spp": lambda: scenes.cornell_box(res=256, spp=16),
    "env_knot_96x54_16spp": lambda: dataclasses.replace(
        scenes.env_knot_small(), params=dataclasses.replace(scenes.env_knot_small().params, spp=16)),
    "inverse_128x128_16spp": lambda: scenes.inverse_box(level=5, res=128, spp=16, max_depth=8, rr_depth=8),
}


def zstat_golden(tmp):
    """Per-pixel mean and variance of the reference's PathTracing::Li over
    samples 0..spp-1 of every pixel (float32), for the per-pixel z-test of
    the GPU's converged image."""
    for name, make in ZSTAT_SCENES.items():
        sd = make()
        path = os.path.join(tmp, "z_%s.gyts" % name)
        io.write_scene(path, sd)
        W, H, S = sd.camera.res_x, sd.camera.res_y, sd.params.spp
        pix = np.repeat(np.arange(W * H), S)
        r = io.ref_paths(tmp, path, pix % W, pix // W, np.tile(np.arange(S), W * H))
        L = r[:, :3].astype(np.float64).reshape(W * H, S, 3)
        np.savez_compressed(os.path.join(HERE, "zstat_%s.npz" % name), mean=L.mean(1).astype(np.float32),
                            var=L.var(1, ddof=1).astype(np.float32), spp=S, res=np.array([W, H]))


def main():
    if sys.argv[1:] == ["zstat"]:
        zstat_golden(tempfile.mkdtemp())
        print("z-test moments written to", HERE)
        return
    if sys.argv[1:] == ["vpt"]:
        volume_golden(tempfile.mkdtemp())
        print("volume golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["vpt_eq"]:
        volume_equi_angular_golden(tempfile.mkdtemp())
        print("equi-angular volume golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["lt"]:
        light_tracing_golden(tempfile.mkdtemp())
        print("light-tracing golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["obj"]:
        obj_golden(tempfile.mkdtemp())
        print("OBJ golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["film"]:
        film_output_golden(tempfile.mkdtemp())
        print("film-output golden vectors written to", HERE)
        return
    if not io.have_harness():
        sys.exit("build the reference harness first: python oracle/ref/build_ref.py")
    tmp = tempfile.mkdtemp()
    if sys.argv[1:] == ["halton"]:
        halton_golden(tmp)
        print("Halton golden vectors written to", HERE)
        return
    rng = np.random.default_rng(20261203)
    out = {}

    # Sobol' points: sobol::sample over dimensions and 64-bit indices
    dims = np.concatenate([rng.integers(0, 1024, 3000), np.arange(16).repeat(8)]).astype(np.uint32)
    idx = np.concatenate([rng.integers(0, 1 << 40, 3000), rng.integers(0, 1 << 20, 128)]).astype(np.uint64)
    np.savez_compressed(os.path.join(HERE, "sobol.npz"), dims=dims, indices=idx,
                        values=io.ref_sobol(tmp, dims, idx))

    # pixel enumeration: SobolEnum::GetIndex at three film sizes
    enum = {}
    for rx, ry in ((256, 256), (1024, 1024), (1920, 1080)):
        s = rng.integers(0, 256, 1500).astype(np.uint32)
        x = rng.integers(0, rx, 1500).astype(np.uint32)
        y = rng.integers(0, ry, 1500).astype(np.uint32)
        key = "%dx%d" % (rx, ry)
        enum[key + "_sxy"] = np.stack([s, x, y], 1)
        enum[key + "_index"] = io.ref_enum(tmp, rx, ry, s, x, y)
    np.savez_compressed(os.path.join(HERE, "enum.npz"), **enum)

    # camera: RasterToWorld of two films
    cams = {}
    for rx, ry in ((256, 256), (1920, 1080)):
        sd = scenes.cornell_box(res=rx, spheres=False)
        sd.camera.res_x, sd.camera.res_y = rx, ry
        path = os.path.join(tmp, "cam.gyts")
        io.write_scene(path, sd)
        cams["%dx%d" % (rx, ry)] = io.ref_camera(tmp, path)
    np.savez_compressed(os.path.join(HERE, "camera.npz"), **cams)

    # closest hits on the Cornell box with spheres and on a small mesh scene
    for name, sd in (("cornell", scenes.cornell_box()), ("mesh", scenes.mixed_materials_box(level=3))):
        path = os.path.join(tmp, name + ".gyts")
        io.write_scene(path, sd)
        rays = random_rays(sd, 3000, rng)
        h = io.ref_hits(tmp, path, rays)
        a = io.ref_hits(tmp, path, rays, any_hit=True)
        np.savez_compressed(os.path.join(HERE, "hits_%s.npz" % name), rays=rays.view(np.float32).reshape(-1, 7),
                            prim=h["prim"], t=h["t"], b1=h["b1"], b2=h["b2"], any=a["prim"])

    # per-path radiance, PathTracing::Li, for three scenes
    for name, sd in (("cornell_nospheres", scenes.cornell_box(spheres=False)), ("cornell", scenes.cornell_box()),
                     ("mixed", scenes.mixed_materials_box(level=3, res=64)), ("env", scenes.env_knot_small())):
        path = os.path.join(tmp, name + ".gyts")
        io.write_scene(path, sd)
        n = 3000
        x = rng.integers(0, sd.camera.res_x, n)
        y = rng.integers(0, sd.camera.res_y, n)
        s = rng.integers(0, sd.params.spp, n)
        r = io.ref_paths(tmp, path, x, y, s)
        np.savez_compressed(os.path.join(HERE, "paths_%s.npz" % name), xys=np.stack([x, y, s], 1).astype(np.uint32),
                            L=r[:, :3], cursor=r[:, 3].astype(np.int32))

    # a full low-resolution render through TiledIntegrator::Render
    sd = scenes.cornell_box(res=64, spp=4)
    path = os.path.join(tmp, "img.gyts")
    io.write_scene(path, sd)
    img, info = io.ref_render(tmp, path)
    np.savez_compressed(os.path.join(HERE, "image_cornell_64x64_4spp.npz"), film=img)

    # a higher-spp render for the statistical image comparison
    sd = scenes.cornell_box(res=128, spp=16)
    path = os.path.join(tmp, "img2.gyts")
    io.write_scene(path, sd)
    img, info = io.ref_render(tmp, path)
    np.savez_compressed(os.path.join(HERE, "image_cornell_128x128_16spp.npz"), film=img)

    # the environment-lit scene through TiledIntegrator::Render
    sd = scenes.env_knot_small()
    path = os.path.join(tmp, "img3.gyts")
    io.write_scene(path, sd)
    img, info = io.ref_render(tmp, path)
    np.savez_compressed(os.path.join(HERE, "image_env_knot_96x54_4spp.npz"), film=img)

    # BxDF tables in the local frame
    cases = bsdf_cases(rng)
    np.savez_compressed(os.path.join(HERE, "bsdf.npz"), cases=cases.view(np.uint8), out=io.ref_bsdf(tmp, cases))
    halton_golden(tmp)
    film_output_golden(tmp)
    obj_golden(tmp)
    light_tracing_golden(tmp)
    volume_golden(tmp)
    volume_equi_angular_golden(tmp)
    zstat_golden(tmp)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
