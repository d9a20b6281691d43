"""The 8-wide compressed BVH (bvh_width=8) against the reference's golden hits,
the oracle and the binary BVH: the same closest hits (up to equal-t ties), the
same occlusion answers and the same paths. Needs a B200."""
import numpy as np
import pytest
import torch

from conftest import golden
import gyunity_b200 as g
from gyunity_b200 import scenes
from oracle.port import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx8():
    c = g.Context(0, bvh_width=8)
    yield c
    c.close()


def _ties(t_gpu, t_ref):
    return np.abs(t_gpu - t_ref) <= 1e-6 * np.maximum(np.abs(t_ref), 1e-6)


def _rays(n, seed, inside=0.95):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-inside, inside, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.3, rng.uniform(0.05, 1.5, n), np.inf).astype(np.float32)
    return np.concatenate([o, d.astype(np.float32), tmax[:, None]], 1)


@pytest.mark.parametrize("name", ["cornell", "mesh"])
def test_wide_closest_hits_match_reference(ctx8, name):
    gd = golden("hits_%s.npz" % name)
    sd = scenes.cornell_box() if name == "cornell" else scenes.mixed_materials_box(level=3)
    sc = g.Scene(sd, ctx8)
    prim, t, _, _ = sc.intersect(gd["rays"])
    ref_t = gd["t"].astype(np.float64)
    same = prim == gd["prim"]
    tie = (prim >= 0) & (gd["prim"] >= 0) & _ties(t, ref_t)
    assert np.all(same | tie), np.nonzero(~(same | tie))[0][:10]
    (occ,) = sc.intersect(gd["rays"], any_hit=True)
    assert np.array_equal(occ, gd["any"].astype(bool))


def test_wide_matches_oracle_and_binary_on_large_mesh(ctx, ctx8):
    # 1.3M-triangle procedural mesh; rays from inside the box, some with a finite tmax
    sd = scenes.procedural_mesh_box(level=8, res=64, spp=1)
    rays = _rays(30000, 11)
    s8, s2 = g.Scene(sd, ctx8), g.Scene(sd, ctx)
    p8, t8, _, _ = s8.intersect(rays)
    p2, t2, _, _ = s2.intersect(rays)
    po, to, _, _ = orc.OracleScene(sd).closest_hit(rays, precision=32)
    for p, t in ((p8, t8), (p2, t2)):
        assert np.all((p == po) | _ties(t, to))
    print("wide vs binary: identical ids", float((p8 == p2).mean()))
    (o8,) = s8.intersect(rays, any_hit=True)
    (o2,) = s2.intersect(rays, any_hit=True)
    assert np.array_equal(o8, o2)
    assert np.array_equal(o8, p2 >= 0)


def test_wide_paths_equal_binary_paths(ctx, ctx8):
    sd = scenes.procedural_mesh_box(level=6, res=48, spp=2)
    n = sd.camera.res_x * sd.camera.res_y * sd.params.spp
    k = np.arange(n)
    xys = np.stack([(k // 2) % 48, (k // 2) // 48, k % 2], 1).astype(np.uint32)
    L8, c8, _ = g.Scene(sd, ctx8).trace_paths(xys)
    L2, c2, _ = g.Scene(sd, ctx).trace_paths(xys)
    same = (c8 == c2) & np.all(L8 == L2, axis=1)
    print("paths identical between the widths:", same.mean())
    assert same.mean() > 0.999


def test_wide_render_equals_binary_render(ctx, ctx8):
    sd = scenes.mixed_materials_box(level=4, res=64, spp=4)
    films = []
    for c in (ctx, ctx8):
        f = torch.zeros(64 * 64 * 4, dtype=torch.float64, device="cuda")
        c.render_device(g.Scene(sd, c), sd.camera, sd.params, f.data_ptr())
        films.append(f.view(64, 64, 4).cpu().numpy())
    assert np.array_equal(films[0][..., 3], films[1][..., 3])
    rel = np.abs(films[0] - films[1]).max() / np.abs(films[0]).max()
    print("largest film difference (relative):", rel)
    assert rel < 1e-3
