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


def _noalloc(ctx, dsc, cam, td, rgb, paths, spp=1):
    import torch
    c = api.camera_struct(cam)
    p = api.params_struct(td, 0.5, spp)
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
