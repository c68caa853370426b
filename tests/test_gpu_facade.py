"""The C++ drop-in facade (include/eos/eos.hpp): a program written like a caller of the
reference renders through DeviceRenderer / RayTracer; its RGBA8 output equals the C ABI's
and the reference renderer's (outside the oracle's flagged paths)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes
from tests.parity import classify, path_mismatch

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp):
    exe = os.path.join(tmp, "facade_render")
    lib = os.path.join(ROOT, "eos_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_render.cpp"), "-o", exe, "-L", lib, "-leos_b200",
           f"-Wl,-rpath,{lib}"]
    subprocess.run(cmd, check=True)
    return exe


def _write_scene(path, sc, cam, td):
    with open(path, "wb") as f:
        np.array([sc.verts.shape[0], sc.n_tris, sc.n_objects, sc.n_lights, cam.width, cam.height, td],
                 np.int32).tofile(f)
        for a in (sc.verts, sc.normals):
            a.astype(np.float32).tofile(f)
        sc.tris.astype(np.uint32).tofile(f)
        sc.tri_obj.astype(np.uint32).tofile(f)
        sc.materials.astype(np.float32).tofile(f)
        sc.lights.astype(np.float32).tofile(f)
        cam.as_array().tofile(f)


def test_cpp_facade_matches_c_abi_and_reference(ctx, tmp_path):
    exe = _build(str(tmp_path))
    sc = scenes.config1_scene()
    cam = scenes.config1_camera(256, 256)
    td = 1
    _write_scene(tmp_path / "scene.bin", sc, cam, td)
    out1, out2, out3 = tmp_path / "dr.rgba", tmp_path / "rt.rgba", tmp_path / "multi.rgba"
    r = subprocess.run([exe, str(tmp_path / "scene.bin"), str(out1), str(out2), str(out3)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    img_dr = np.fromfile(out1, np.uint8).reshape(cam.height, cam.width, 4)
    img_rt = np.fromfile(out2, np.uint8).reshape(cam.height, cam.width, 4)
    img_multi = np.fromfile(out3, np.uint8).reshape(cam.height, cam.width, 4)
    assert np.array_equal(img_dr, img_rt)
    assert np.array_equal(img_dr, img_multi)  # split-frame bands, one context each
    dsc = api.DeviceScene(ctx, sc)
    g = api.render(ctx, dsc, cam, td, pixel_offset=0.0, outputs=("rgba8",), device=False)
    assert np.array_equal(img_dr, g["rgba8"])
    if oracle.ref_available():
        ref = oracle.RefRenderer(sc)
        img_ref, _ = ref.render_rgba8(cam, td)
        rr = ref.render(cam, td, pixel_offset=0.0)
        o = oracle.Oracle(sc).render(cam, td, pixel_offset=0.0)
        mm = path_mismatch(o["hits"], o["shadows"], rr["hits"], rr["shadows"], td + 1)
        c = classify(mm, o["flags"])
        assert c["unexplained"] == 0
        differ = (img_dr.reshape(-1, 4) != img_ref.reshape(-1, 4)).any(1)
        # equal 8-bit output outside flagged paths, but for colours that land within an
        # ulp of a quantisation step (powf of the GPU vs glibc)
        assert (differ & ~mm).sum() <= 0.001 * mm.size
