"""OBJ ingestion on the CPU (gyt_mesh_load_obj, host code) against the
reference's Mesh::LoadFromFile compiled from its sources
(tests/golden/obj_meshes.npz over tests/golden/obj/*.obj): bit-exact
positions and normals for triangles, polygons (ear clipping), every face-index
form, number format and line ending, both vertex orders. The transform
composition (gyunity_b200.mesh.Transform) is checked through a float32
restatement of Triangle::SetTransform; the GPU step itself is in
test_gpu_obj.py."""
import os

import numpy as np
import pytest

from conftest import golden
from gyunity_b200.mesh import Mesh, Transform
from gyunity_b200._capi import GytError

HERE = os.path.dirname(os.path.abspath(__file__))
OBJ = os.path.join(HERE, "golden", "obj")
NAMES = ["polygons", "forms", "generated_normals", "sphere"]
F = np.float32


def _bits(a):
    return np.ascontiguousarray(a, F).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("rev", [0, 1])
def test_loader_bit_exact(name, rev):
    ref = golden("obj_meshes.npz")["%s_rev%d" % (name, rev)]
    p, n, _ = Mesh.load_obj(os.path.join(OBJ, name + ".obj"), rev).arrays()
    assert p.shape[0] == ref.shape[0]
    assert np.array_equal(_bits(p), _bits(ref[:, :3]))
    assert np.array_equal(_bits(n), _bits(ref[:, 3:]))


def transform_from_spec(spec):
    t = Transform()
    for item in spec.split(";"):
        op, *a = item.split()
        a = [float(x) for x in a]
        if op == "T":
            u = Transform.Translate(a)
        elif op == "S":
            u = Transform.Scale(*a)
        else:
            u = {"RX": Transform.RotateX, "RY": Transform.RotateY, "RZ": Transform.RotateZ}[op](a[0])
        t = t * u
    return t


def set_transform(t, p, n):
    """Triangle::SetTransform in float32, the reference's operation order."""
    m, inv = t.m, t.inv
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    r = []
    for k in range(4):
        a = m[k, 3]
        a = m[k, 2] * z + a
        a = m[k, 1] * y + a
        r.append(m[k, 0] * x + a)
    P = np.stack(r[:3], -1)
    w = r[3]
    P = np.where(((w == 1) | (w == 0))[..., None], P, P / w[..., None])
    q = []
    for k in range(3):
        a = inv[3, k] * F(0)
        a = inv[2, k] * n[..., 2] + a
        a = inv[1, k] * n[..., 1] + a
        q.append(inv[0, k] * n[..., 0] + a)
    q = np.stack(q, -1)
    ln = np.sqrt((q[..., 0] * q[..., 0] + q[..., 1] * q[..., 1]) + q[..., 2] * q[..., 2])
    return P, q / ln[..., None]


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("k", [0, 1, 2])
def test_transform_composition_bit_exact(name, k):
    g = golden("obj_meshes.npz")
    ref = g["%s_t%d" % (name, k)]
    p, n, _ = Mesh.load_obj(os.path.join(OBJ, name + ".obj")).arrays()
    with np.errstate(all="ignore"):
        P, N = set_transform(transform_from_spec(str(g["transforms"][k])), p, n)
    assert np.array_equal(_bits(P), _bits(ref[:, :3]))
    ok = np.all(np.isfinite(ref[:, 3:]), axis=-1)  # zero-area faces keep an unnormalisable normal
    assert np.array_equal(_bits(N)[ok], _bits(ref[:, 3:])[ok])


def test_polygon_triangulation_counts():
    # 12 quads -> 24, the pentagon -> 3, the concave hexagon -> 4, the quad
    # with three collinear vertices -> 2
    p, _, _ = Mesh.load_obj(os.path.join(OBJ, "polygons.obj")).arrays()
    assert p.shape == (33, 3, 3)


@pytest.mark.parametrize("text,why", [("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n", "zero index"),
                                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", "out of range"),
                                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2 3\n", "partial normals")])
def test_malformed_files_fail_with_a_message(tmp_path, text, why):
    path = tmp_path / "bad.obj"
    path.write_text(text)
    with pytest.raises(GytError) as e:
        Mesh.load_obj(str(path))
    assert "bad.obj" in str(e.value), why
    with pytest.raises(GytError):
        Mesh.load_obj(str(tmp_path / "missing.obj"))


def _reference_meshes():
    from oracle.ref.build_ref import DEFAULT_REFERENCE
    return os.path.join(DEFAULT_REFERENCE, "resources", "meshs")


@pytest.mark.skipif(not os.path.isdir(_reference_meshes()), reason="needs the reference checkout")
def test_reference_assets_load_like_the_reference(tmp_path):
    # the reference's own meshes (not part of this repository), where present
    from oracle import scene_io as io
    if not io.have_harness():
        pytest.skip("reference harness not built")
    for name in ("cube.obj", "bunny.obj", "water.obj"):
        path = os.path.join(_reference_meshes(), name)
        ref = io.ref_obj(str(tmp_path), path, 0, "-")
        p, n, _ = Mesh.load_obj(path).arrays()
        assert np.array_equal(_bits(p), _bits(ref[:, :3])) and np.array_equal(_bits(n), _bits(ref[:, 3:])), name
