"""Meshes read from OBJ files render through the GPU path exactly as the oracle renders
the same triangles, in plain and batched mode; the C++ facade's TriangleMesh (the
reference's loadFromFile / addTriangleMesh flow) gives the same image as the C ABI."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from eos_b200 import api, mesh, scenes
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MESHES = os.path.join(HERE, "golden", "meshes")


def _paths(p):
    return p[:, :8], p[:, 8:].view(np.uint32)


def _mesh_scene():
    blob = mesh.load_obj(os.path.join(MESHES, "blob.obj"))
    shapes = mesh.load_obj(os.path.join(MESHES, "shapes.obj"))
    grid = mesh.load_obj(os.path.join(MESHES, "grid_vn.obj"))
    parts = [mesh.transform(blob, M) for M in (np.diag([1.0, 1.0, 1.0, 1.0]),
                                                np.array([[0.6, 0, 0, 2.2], [0, 0.6, 0, 0.3], [0, 0, 0.6, -0.5],
                                                          [0, 0, 0, 1]]))]
    parts.append(mesh.transform(shapes, np.array([[0.4, 0, 0, -2.5], [0, 0.4, 0, -0.2], [0, 0, 0.4, 0.3],
                                                  [0, 0, 0, 1]])))
    parts.append(mesh.transform(grid, np.array([[3, 0, 0, 0], [0, 1, 0, -1.3], [0, 0, 3, 0], [0, 0, 0, 1]])))
    mats = np.array([[0.8, 0.3, 0.3, 0.4, 0.4, 0.4, 32, 0.2],
                     [0.2, 0.7, 0.3, 0.3, 0.3, 0.3, 64, 0.0],
                     [0.3, 0.3, 0.9, 0.5, 0.5, 0.5, 16, 0.5],
                     [0.6, 0.6, 0.6, 0.1, 0.1, 0.1, 8, 0.3]], np.float32)
    lights = np.array([[5, 5, 5, 1, 1, 1], [-4, 3, 2, 0.6, 0.7, 0.9]], np.float32)
    return mesh.scene_from_meshes(parts, mats, lights, name="obj meshes")


def test_obj_scene_matches_oracle(ctx):
    sc = _mesh_scene()
    cam = scenes.look_at((0.5, 2.0, 6.0), (0, -0.3, 0), 50.0, 160, 120)
    o = oracle.Oracle(sc).render(cam, 3, pixel_offset=0.5)
    dsc = api.DeviceScene(ctx, sc)
    for mode in ("plain", "wavefront"):
        g = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, mode=mode, outputs=("rgb", "paths"), device=False)
        gh, gs = _paths(g["paths"])
        assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"]), mode
        assert np.abs(g["rgb"] - o["rgb"]).max() <= RGB_TOL, mode
    assert (o["hits"][:, 0] >= 0).sum() > 0.3 * cam.width * cam.height


def test_facade_triangle_mesh_matches_c_abi(ctx, tmp_path):
    exe = str(tmp_path / "facade_mesh")
    lib = os.path.join(ROOT, "eos_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_mesh.cpp"), "-o", exe, "-L", lib, "-leos_b200",
                    f"-Wl,-rpath,{lib}"], check=True)
    path = os.path.join(MESHES, "blob.obj")
    cam = scenes.look_at((0.3, 1.2, 3.5), (0, 0, 0), 45.0, 96, 80)
    td = 2
    out = tmp_path / "img.rgba"
    r = subprocess.run([exe, path, str(out), str(cam.width), str(cam.height), str(td)]
                       + [repr(float(x)) for x in cam.as_array()], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "triangles 1280" in r.stdout
    img = np.fromfile(out, np.uint8).reshape(cam.height, cam.width, 4)
    m = mesh.load_obj(path)
    sc = mesh.scene_from_meshes([m], [[0.87, 0.3, 0.5, 1, 1, 1, 120, 0.25]],
                                [[5, 5, 5, 1, 1, 1], [-4, 3, 2, 0.6, 0.7, 0.9]])
    g = api.render(ctx, api.DeviceScene(ctx, sc), cam, td, pixel_offset=0.0, outputs=("rgba8",), device=False)
    assert np.array_equal(img, g["rgba8"])
    assert (img[..., :3].reshape(-1, 3).sum(1) > 0).sum() > 100
