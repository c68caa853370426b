"""OBJ ingestion (eos_mesh_*; host code, no GPU): the library's C++ loader equals the
Python restatement of assimp's import steps (oracle/mesh_oracle.py) bit for bit on the
generated fixtures (tests/golden/meshes, from tests/golden/make_meshes.py) and, when the
reference tree is present, on the reference's own sample models; plus the semantics of
each step and the error statuses."""
import glob
import os

import numpy as np
import pytest

from eos_b200 import mesh
from eos_b200._lib import EosError
import oracle
from oracle import mesh_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "meshes", "*.obj")))
REF_MODELS = os.path.join(oracle.REF_ROOT, "objmodels")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _same(m, o):
    v, n, t, nf, nfaces = o
    return (np.array_equal(_bits(m.verts), _bits(v)) and np.array_equal(_bits(m.normals), _bits(n))
            and np.array_equal(m.tris, t) and m.normals_from_file == bool(nf) and m.n_faces == nfaces)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_loader_matches_restatement(path):
    m = mesh.load_obj(path)
    with open(path, newline="") as f:
        assert _same(m, mesh_oracle.parse_obj(f.read()))
    # the same text from memory gives the same mesh
    with open(path, "rb") as f:
        m2 = mesh.parse_obj(f.read())
    assert np.array_equal(m2.tris, m.tris) and np.array_equal(_bits(m2.normals), _bits(m.normals))


def test_step_semantics():
    d = os.path.join(HERE, "golden", "meshes")
    blob = mesh.load_obj(os.path.join(d, "blob.obj"))
    # generated normals are unit vectors, one per distinct position (the repeated cap
    # vertices are joined back): the level-3 icosphere's 642 vertices
    assert not blob.normals_from_file and blob.verts.shape[0] == 642 and blob.n_tris == 1280
    assert np.abs(np.linalg.norm(blob.normals, axis=1) - 1).max() < 1e-6
    # smooth normals point outwards on a star-shaped blob
    assert (np.einsum("ij,ij->i", blob.normals, blob.verts) > 0).all()

    shapes = mesh.load_obj(os.path.join(d, "shapes.obj"))
    assert shapes.n_faces == 9 and shapes.n_tris == 6 * 2 + 2 + 3  # box quads, arrow, pentagon; line dropped
    V = shapes.verts
    arrow = shapes.tris[12:14]
    # the concave quad is fanned from its reflex corner (4, 0.5, 0)
    assert np.allclose(V[arrow[0, 0]], [4, 0.5, 0]) and np.allclose(V[arrow[1, 0]], [4, 0.5, 0])
    # both arrow triangles lie inside the polygon: their areas sum to the polygon's area
    def area(t):
        a, b, c = V[t[0]], V[t[1]], V[t[2]]
        return 0.5 * np.linalg.norm(np.cross(b - a, c - a))
    assert abs(area(arrow[0]) + area(arrow[1]) - 1.25) < 1e-6

    grid = mesh.load_obj(os.path.join(d, "grid_vn.obj"))
    assert grid.normals_from_file and grid.n_faces == 36 and grid.n_tris == 48

    near = mesh.load_obj(os.path.join(d, "near.obj"))
    N = near.normals[near.tris.reshape(-1)]
    # corners (0,0,0) and (0.001,0,0) are within the smoothing distance: same normal;
    # (0,0.003,0) is not
    assert np.array_equal(N[0], N[3]) and not np.array_equal(N[0], N[6])


@pytest.mark.parametrize("text,code", [
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n", 10),   # index out of range
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 x\n", 10),   # not a number
    ("v 0 0\n", 10),                                # short vertex
    ("# nothing\n", 10),                            # no triangles
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n", 10),     # only a line
])
def test_malformed_input_reports_parse_error(text, code):
    with pytest.raises(EosError) as e:
        mesh.parse_obj(text)
    assert e.value.code == code


def test_missing_file_reports_io_error(tmp_path):
    with pytest.raises(EosError) as e:
        mesh.load_obj(str(tmp_path / "missing.obj"))
    assert e.value.code == 9


def test_negative_indices_and_normals():
    text = "v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf -3//-1 -2//-1 -1//-1\n"
    m = mesh.parse_obj(text)
    assert m.normals_from_file and m.n_tris == 1
    assert np.array_equal(m.verts[m.tris[0]], np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32))
    assert np.array_equal(m.normals, np.tile(np.array([[0, 0, 1]], np.float32), (3, 1)))


def test_scene_from_meshes_object_ids():
    d = os.path.join(HERE, "golden", "meshes")
    a = mesh.load_obj(os.path.join(d, "blob.obj"))
    b = mesh.transform(mesh.load_obj(os.path.join(d, "shapes.obj")), np.diag([1.0, 2.0, 1.0, 1.0]))
    mats = np.tile(np.array([0.5, 0.5, 0.5, 0.2, 0.2, 0.2, 16, 0.0], np.float32), (2, 1))
    sc = mesh.scene_from_meshes([a, b], mats, [[5, 5, 5, 1, 1, 1]])
    assert sc.n_tris == a.n_tris + b.n_tris
    assert (sc.tri_obj[:a.n_tris] == 0).all() and (sc.tri_obj[a.n_tris:] == 1).all()
    assert sc.tris.max() == a.verts.shape[0] + b.verts.shape[0] - 1


@pytest.mark.skipif(not os.path.isdir(REF_MODELS), reason="reference tree not present")
@pytest.mark.parametrize("name", ["grid.obj", "grid_back.obj", "triangle_grid.obj", "monkey.obj", "head.obj"])
def test_reference_models_match_restatement(name):
    path = os.path.join(REF_MODELS, name)
    m = mesh.load_obj(path)
    with open(path, newline="") as f:
        assert _same(m, mesh_oracle.parse_obj(f.read()))
    assert np.abs(np.linalg.norm(m.normals, axis=1) - 1).max() < 1e-5


@pytest.mark.skipif(not os.path.isdir(REF_MODELS), reason="reference tree not present")
def test_reference_bunny_loads():
    m = mesh.load_obj(os.path.join(REF_MODELS, "bunny.obj"))
    assert m.n_tris == 69666 and not m.normals_from_file
    assert np.isfinite(m.normals).all()
