"""Procedural workload generators: sizes, determinism, layout."""
import numpy as np

from gyunity_b200 import scenes


def test_cornell_box_layout():
    sd = scenes.cornell_box()
    assert sd.n_triangles == 12 and sd.n_spheres == 2
    assert (sd.tri_emission >= 0).sum() == 2
    assert sd.n_paths() == 256 * 256 * 16
    # walls face inwards: the shading normal points into the box
    v = sd.vertices[sd.indices]
    c = v.mean(1)
    n = sd.normals[sd.indices[:, 0]]
    assert np.all(np.einsum("ij,ij->i", n, -c) > 0)


def test_icosphere_counts():
    for level in range(0, 5):
        v, f = scenes.icosphere(level)
        assert f.shape[0] == 20 * 4 ** level
        assert v.shape[0] == 10 * 4 ** level + 2


def test_procedural_mesh_is_deterministic():
    a = scenes.procedural_mesh_box(level=4, res=64, spp=2)
    b = scenes.procedural_mesh_box(level=4, res=64, spp=2)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.mat_params, b.mat_params)
    r = np.linalg.norm(a.vertices[12 * 0 + 24:] - np.array([0, -0.55, 0], np.float32), axis=1)
    assert np.all(np.abs(r - 0.4) <= 0.05 * 0.4 + 1e-5)
    alphas = a.mat_params[a.mat_type == scenes.MAT_CONDUCTOR][:, 6]
    assert alphas.shape[0] == 64 and np.all((alphas >= 0.05) & (alphas <= 0.5))


def test_roughness_to_alpha():
    assert abs(scenes.roughness_to_alpha(0.5) - 1.62142 - 0.819955 * np.log(0.5) - 0.1734 * np.log(0.5) ** 2
               - 0.0171201 * np.log(0.5) ** 3 - 0.000640711 * np.log(0.5) ** 4) < 1e-5


def test_cornell_fog_layout():
    sd = scenes.cornell_fog(res=32, spp=2)
    nt = sd.n_triangles
    assert nt == 14 and sd.media.shape == (1, 7) and sd.tri_medium.shape == (nt, 2)
    # only the front quad is a medium boundary, and it has no material
    inside = np.nonzero(sd.tri_medium[:, 0] >= 0)[0]
    assert list(inside) == [12, 13]
    assert np.all(sd.mat_type[sd.tri_material[inside]] == scenes.MAT_NONE)
    assert np.all(sd.tri_medium[:12] == -1) and np.all(sd.tri_medium[12:, 1] == -1)
    assert np.all(sd.vertices[sd.indices[12:]][..., 2] == 1.0)


def test_fog_ball_layout():
    sd = scenes.fog_ball_box(level=2)
    ball = np.arange(12, sd.n_triangles)
    assert ball.shape[0] == 320 and sd.media.shape == (1, 7)
    assert np.all(sd.tri_medium[ball] == (0, -1)) and np.all(sd.tri_medium[:12] == -1)
    assert np.all(sd.mat_type[sd.tri_material[ball]] == scenes.MAT_NONE)
    # outward shading normals: leaving along the normal enters the outside (no medium)
    c = sd.vertices[sd.indices[ball]].mean(1) - np.array([0.0, -0.45, 0.0])
    assert np.all(np.einsum("ij,ij->i", c, sd.normals[sd.indices[ball, 0]]) > 0)
