"""The device BVH builder against the host builder (both replace BVHAccel's
build, accelerator/BVHAccel.cpp:154-372): the same tree (splits, leaf sets,
child boxes bit for bit), the same hits and the same image. Needs a B200."""
import dataclasses

import numpy as np
import pytest

from bvh_tools import canonical, leaf_orders, validate
import gyunity_b200 as g
from gyunity_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx_host():
    c = g.Context(0, bvh_builder="host")
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_dev():
    c = g.Context(0, bvh_builder="device")
    yield c
    c.close()


def _with_triangles(sd, v, idx):
    """The scene's materials and camera with other triangles (no lights)."""
    nt = idx.shape[0]
    return dataclasses.replace(sd, vertices=np.ascontiguousarray(v, np.float32),
                               indices=np.ascontiguousarray(idx, np.uint32), normals=None,
                               tri_material=np.zeros(nt, np.uint32), tri_emission=np.full(nt, -1, np.int32))


def _random_soup(n, seed, size=0.05):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.9, 0.9, (n, 1, 3))
    v = (c + rng.uniform(-size, size, (n, 3, 3))).reshape(-1, 3)
    return v, np.arange(3 * n, dtype=np.uint32).reshape(n, 3)


def _scene_cases():
    base = scenes.cornell_box(res=32, spp=1, spheres=False)
    cases = {"cornell": base}
    for n in (1, 2, 5, 8, 9, 33, 100, 4097):
        v, i = _random_soup(n, seed=n)
        cases["soup%d" % n] = _with_triangles(base, v, i)
    # 40 copies of one triangle among 60 others: a task whose centroids all coincide
    v, i = _random_soup(60, seed=3)
    same = np.array([[0.1, 0.2, 0.3], [0.2, 0.25, 0.3], [0.15, 0.3, 0.35]], np.float32)
    v = np.concatenate([v, np.tile(same, (40, 1))])
    cases["coincident"] = _with_triangles(base, v, np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3))
    cases["mesh_l5"] = scenes.procedural_mesh_box(level=5, res=32, spp=1)
    return cases


CASES = _scene_cases()


@pytest.mark.parametrize("name", list(CASES))
def test_device_tree_is_valid(ctx_dev, name):
    sd = CASES[name]
    sc = g.Scene(sd, ctx_dev)
    nodes, ids = sc.read_bvh()
    inner, depth = validate(nodes, ids, sd.vertices, sd.indices)
    assert inner == sc.info()["bvh_nodes"]
    assert depth < 64


@pytest.mark.parametrize("name", [n for n in CASES if n != "coincident"])
def test_device_tree_equals_host_tree(ctx_host, ctx_dev, name):
    sd = CASES[name]
    a = g.Scene(sd, ctx_host).read_bvh()
    b = g.Scene(sd, ctx_dev).read_bvh()
    ca, cb = canonical(*a), canonical(*b)
    assert len(ca) == len(cb)
    assert ca == cb
    assert leaf_orders(*a) == leaf_orders(*b)


def test_device_tree_equals_host_tree_large(ctx_host, ctx_dev):
    # 1.3M triangles: the bench scene
    sd = scenes.procedural_mesh_box(level=8, res=64, spp=1)
    ha = g.Scene(sd, ctx_host)
    hb = g.Scene(sd, ctx_dev)
    assert ha.info()["bvh_nodes"] == hb.info()["bvh_nodes"]
    assert canonical(*ha.read_bvh()) == canonical(*hb.read_bvh())


def test_same_hits_both_builders(ctx_host, ctx_dev):
    sd = CASES["mesh_l5"]
    rng = np.random.default_rng(11)
    n = 20000
    o = rng.uniform(-0.95, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d.astype(np.float32), np.full((n, 1), np.inf, np.float32)], 1)
    pa, ta, ua, va = g.Scene(sd, ctx_host).intersect(rays)
    pb, tb, ub, vb = g.Scene(sd, ctx_dev).intersect(rays)
    # same tree and the same triangle order in every leaf: identical results
    assert np.array_equal(pa, pb)
    assert np.array_equal(ta, tb) and np.array_equal(ua, ub) and np.array_equal(va, vb)
    (aa,) = g.Scene(sd, ctx_host).intersect(rays, any_hit=True)
    (ab,) = g.Scene(sd, ctx_dev).intersect(rays, any_hit=True)
    assert np.array_equal(aa, ab)


def test_same_image_both_builders(ctx_host, ctx_dev):
    sd = scenes.procedural_mesh_box(level=5, res=64, spp=4, max_depth=8)
    imgs = []
    for c in (ctx_host, ctx_dev):
        sc = g.Scene(sd, c)
        cam = g.PinHoleCamera(g.Film(64, 64), sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy,
                              sd.camera.film_distance)
        film = g.GpuPathTracing(sd.params.spp, sd.params.max_depth, sd.params.rr_depth).Render(sc, cam)
        imgs.append(film.GetImage())
    a, b = imgs
    # identical paths; only the order of the FP64 film atomics differs
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-12)


def test_builder_option_checked(ctx_dev):
    lib = ctx_dev._lib
    assert lib.gyt_context_set_bvh_builder(ctx_dev.handle, 7) == 1


# ---- the 8-wide BVH: collapse on the device ----------------------------------

@pytest.fixture(scope="module")
def ctx_host8():
    c = g.Context(0, bvh_width=8, bvh_builder="host")
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_dev8():
    c = g.Context(0, bvh_width=8, bvh_builder="device")
    yield c
    c.close()


WIDE_CASES = dict(CASES)
for _n in (3, 4, 17, 40):
    _v, _i = _random_soup(_n, seed=100 + _n)
    WIDE_CASES["soup%d" % _n] = _with_triangles(CASES["cornell"], _v, _i)


@pytest.mark.parametrize("name", list(WIDE_CASES))
def test_device_wide_bvh_equals_host_word_for_word(ctx_host8, ctx_dev8, name):
    """The device collapse gives the host's 8-wide nodes exactly (quantized
    boxes, slot order, child and triangle offsets, breadth-first numbering)
    and the same leaf-order triangles. In the coincident-centroid scene the
    binary builders split the 40 identical triangles by index position, in
    different orders (the binary test above checks that tree for validity
    only): there the nodes are equal and the leaf order is a permutation."""
    sd = WIDE_CASES[name]
    wa, ia = g.Scene(sd, ctx_host8).read_wide_bvh()
    wb, ib = g.Scene(sd, ctx_dev8).read_wide_bvh()
    assert wa.shape == wb.shape and wa.shape[0] >= 1
    assert np.array_equal(wa, wb), np.nonzero((wa != wb).any(1))[0][:10]
    if name == "coincident":
        assert np.array_equal(np.sort(ib), np.arange(sd.n_triangles))
    else:
        assert np.array_equal(ia, ib)


def test_device_wide_bvh_large_and_fast(ctx_host8, ctx_dev8):
    """The 1.31M-triangle procedural mesh: word-for-word equal, built on the
    device (binary build plus collapse) in well under a tenth of a second."""
    import time
    sd = scenes.procedural_mesh_box(level=8, res=64, spp=1)
    # the first build of this size in a process also pays one-time costs
    # (kernel loading, device memory growth: 0.4-1.8 s seen in a fresh
    # process, 0.04 s after other large builds): time the second
    t0 = time.perf_counter()
    g.Scene(sd, ctx_dev8).close()
    first = time.perf_counter() - t0
    t0 = time.perf_counter()
    sb = g.Scene(sd, ctx_dev8)
    dt = time.perf_counter() - t0
    print("first device build in this process: %.3f s" % first)
    t0 = time.perf_counter()
    sa = g.Scene(sd, ctx_host8)
    ht = time.perf_counter() - t0
    wa, ia = sa.read_wide_bvh()
    wb, ib = sb.read_wide_bvh()
    print("8-wide BVH of %d triangles: %d nodes; scene upload and build %.3f s on the device, %.3f s on the host" %
          (sd.n_triangles, wb.shape[0], dt, ht))
    assert np.array_equal(wa, wb) and np.array_equal(ia, ib)
    assert dt < 0.25
