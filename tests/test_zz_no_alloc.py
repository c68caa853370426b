"""eos_render_noalloc: the render entry point that allocates no device memory.

Some callers cannot call cudaMalloc while they render -- code running under another
framework's allocator or memory pool, real-time loops that forbid allocation after
start-up.  For them the library keeps the wavefront queues in one fixed device array and
takes only the scene, the camera, a stream and device output buffers.  This test calls it
through the C ABI twice in a row and compares each result with eos_render, the entry point
that uses context scratch memory.  It lives in its own file, collected last, and passes
both alone in a fresh process and after the other tests.
"""
import ctypes
from ctypes import byref

import numpy as np
import pytest

from eos_b200 import _lib as L
from eos_b200 import api, scenes
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu


def _noalloc(ctx, dsc, cam, td, rgb, paths, spp=1, rows=None, jitter_seed=0, flags=0):
    import torch
    c = api.camera_struct(cam)
    p = api.params_struct(td, 0.5, spp, jitter_seed, rows=rows)
    p.flags = flags
    st = L.Stats()
    stream = torch.cuda.current_stream().cuda_stream
    code = ctx.lib.eos_render_noalloc(dsc.h, byref(c), byref(p), ctypes.c_void_p(stream),
                                      ctypes.c_void_p(rgb.data_ptr()) if rgb is not None else None,
                                      ctypes.c_void_p(paths.data_ptr()) if paths is not None else None, byref(st))
    return code, st


def test_noalloc_matches_render_on_two_calls_in_a_row(ctx):
    import torch
    sc = scenes.small_random_scene(61, n_spheres=6, level=3, lights=3, refl=0.6)
    dsc = api.DeviceScene(ctx, sc)
    cams = [scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 128, 96),
            scenes.look_at((-6.0, 4.0, 6.0), (0, -0.5, 0), 50.0, 120, 100)]
    for i, cam in enumerate(cams):
        npx = cam.width * cam.height
        rgb = torch.full((npx, 3), -1.0, device="cuda")
        paths = torch.zeros((npx, 16), dtype=torch.int32, device="cuda")
        code, st = _noalloc(ctx, dsc, cam, 2, rgb, paths)
        assert code == 0, (i, code)
        torch.cuda.synchronize()
        ref = api.render(ctx, dsc, cam, 2, pixel_offset=0.5, outputs=("rgb", "paths"), device=True)
        assert np.abs(rgb.cpu().numpy() - ref["rgb"].cpu().numpy()).max() <= RGB_TOL
        assert np.array_equal(paths.cpu().numpy(), ref["paths"].cpu().numpy())
        assert st.primary_rays == ref["stats"]["primary_rays"] == npx
        assert st.shadow_rays == ref["stats"]["shadow_rays"]
        assert st.secondary_rays == ref["stats"]["secondary_rays"]


def test_noalloc_rejects_sizes_beyond_its_capacity(ctx):
    import torch
    sc = scenes.small_random_scene(62, n_spheres=3, level=2, lights=2)
    dsc = api.DeviceScene(ctx, sc)
    big = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 256, 256)  # 65,536 paths > 16,384
    rgb = torch.zeros((256 * 256, 3), device="cuda")
    code, _ = _noalloc(ctx, dsc, big, 1, rgb, None)
    assert code == 1
    assert L.NOALLOC_MAX_PATHS == 16384
    # host output buffers are refused too
    small = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 64, 64)
    host = np.zeros((64 * 64, 3), np.float32)
    c = api.camera_struct(small)
    p = api.params_struct(1, 0.5, 1)
    assert ctx.lib.eos_render_noalloc(dsc.h, byref(c), byref(p), None, host.ctypes.data_as(ctypes.c_void_p),
                                      None, None) == 1
    # and a request within the limit still works afterwards
    rgb2 = torch.zeros((64 * 64, 3), device="cuda")
    code, st = _noalloc(ctx, dsc, small, 1, rgb2, None)
    assert code == 0 and st.primary_rays == 64 * 64


def _check_against_render(ctx, dsc, cam, td, spp=1, rows=None, jitter_seed=0):
    """Two calls in a row of the allocation-free entry point against eos_render (wavefront
    mode, context scratch) on the same frame: paths bit for bit, colours within RGB_TOL."""
    import torch
    H = rows[1] - rows[0] if rows else cam.height
    npx = cam.width * H
    ref = api.render(ctx, dsc, cam, td, pixel_offset=0.5, spp=spp, jitter_seed=jitter_seed, mode="wavefront",
                     outputs=("rgb", "paths"), device=True, rows=rows)
    for call in range(2):
        rgb = torch.full((npx, 3), -1.0, device="cuda")
        paths = torch.zeros((npx * spp, 16), dtype=torch.int32, device="cuda")
        code, st = _noalloc(ctx, dsc, cam, td, rgb, paths, spp=spp, rows=rows, jitter_seed=jitter_seed)
        assert code == 0, (call, code)
        torch.cuda.synchronize()
        assert np.abs(rgb.cpu().numpy() - ref["rgb"].cpu().numpy()).max() <= RGB_TOL, call
        assert np.array_equal(paths.cpu().numpy(), ref["paths"].cpu().numpy()), call
        assert st.primary_rays == ref["stats"]["primary_rays"] == npx * spp
        assert st.shadow_rays == ref["stats"]["shadow_rays"]
        assert st.secondary_rays == ref["stats"]["secondary_rays"]


def test_noalloc_two_samples_per_pixel(ctx):
    sc = scenes.small_random_scene(63, n_spheres=5, level=3, lights=2, refl=0.5, transparent=1)
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 96, 80)  # 2 x 7,680 paths <= 16,384
    _check_against_render(ctx, dsc, cam, 3, spp=2, jitter_seed=77)


def test_noalloc_row_band(ctx):
    sc = scenes.small_random_scene(64, n_spheres=6, level=3, lights=3, refl=0.6)
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 320, 240)  # the whole frame is too large,
    _check_against_render(ctx, dsc, cam, 2, rows=(101, 141))             # a 40-row band fits


def test_noalloc_instanced_scene(ctx):
    d = scenes.instanced_test_scene(11, n_instances=8, lights=2, transparent=1)
    meshes = [api.DeviceScene(ctx, m) for m in d.meshes]
    inst = api.InstancedScene(ctx, meshes, d.instances, d.materials, d.lights)
    cam = scenes.look_at((1.0, 3.0, 9.0), (0, 0, 0), 50.0, 128, 96)
    _check_against_render(ctx, inst, cam, 2)


def test_noalloc_refuses_unknown_flags(ctx):
    import torch
    sc = scenes.small_random_scene(65, n_spheres=2, level=2, lights=1)
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 32, 32)
    rgb = torch.zeros((32 * 32, 3), device="cuda")
    for bad in (8, 1 << 30):
        code, _ = _noalloc(ctx, dsc, cam, 1, rgb, None, flags=bad)
        assert code == 1, bad
    code, _ = _noalloc(ctx, dsc, cam, 1, rgb, None, flags=L.FLAG_TREE_RECORDS)  # needs ray-tree queues
    assert code == 7
    code, st = _noalloc(ctx, dsc, cam, 1, rgb, None, flags=1)  # stage timing is accepted and ignored
    assert code == 0 and st.primary_rays == 32 * 32
    code, st = _noalloc(ctx, dsc, cam, 1, rgb, None, spp=4, flags=L.FLAG_AA_GRID)  # the reference's 2x2 grid
    assert code == 0 and st.primary_rays == 4 * 32 * 32
