"""The reference's anti-aliasing grid (RayTracer::setAASamples / renderWithAA,
src/RayTracer.cpp:176-265) on the GPU with EOS_FLAG_AA_GRID: n x n samples per pixel at
(p, q) / n, the pixel their sum times (1/n)^2.  Against the reference's own output (golden
aa3_small12.npz: per-sample paths, FP32 colours and its RGBA8 frame), in plain, wavefront
and batched mode, and the adjoint against the FP64 adjoint on the same grid."""
import os

import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes
from eos_b200._lib import EosError
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _scene():
    return scenes.small_random_scene(12, n_spheres=5, level=2, lights=3, refl=0.6)


@pytest.mark.parametrize("mode", ["plain", "wavefront", "batch"])
def test_aa_grid_matches_reference_golden(ctx, mode):
    gd = np.load(os.path.join(GOLDEN, "aa3_small12.npz"))
    W, H, td, n = (int(v) for v in gd["size"])
    cam = scenes.CameraData(*[gd["cam"][3 * i:3 * i + 3] for i in range(4)], W, H)
    dsc = api.DeviceScene(ctx, _scene())
    if mode == "batch":
        jobs = [api.BatchJob(dsc, cam, td, 0.0, n * n)]
        outs = api.make_batch_outputs(jobs, ("rgb", "rgba8", "paths"))
        st = api.render_batch(ctx, jobs, outs, aa_grid=True)
        rgb, q, paths = (outs[0][k].cpu().numpy() for k in ("rgb", "rgba8", "paths"))
    else:
        r = api.render(ctx, dsc, cam, td, pixel_offset=0.0, spp=n * n, mode=mode,
                       outputs=("rgb", "rgba8", "paths"), device=False, aa_grid=True)
        rgb, q, paths, st = r["rgb"], r["rgba8"], r["paths"], r["stats"]
    assert np.array_equal(paths[:, :td + 1], gd["hits"])
    assert np.array_equal(paths[:, 8:8 + td + 1].view(np.uint32), gd["shadows"])
    assert np.abs(rgb - gd["rgb"]).max() <= RGB_TOL
    assert (rgb == gd["rgb"]).mean() > 0.99
    assert (q[..., :3] != gd["rgba8"][..., :3]).any(-1).mean() <= 0.001
    assert (st["primary_rays"], st["shadow_rays"], st["secondary_rays"]) == tuple(int(v) for v in gd["counts"])


def test_aa_grid_needs_a_square_sample_count(ctx):
    dsc = api.DeviceScene(ctx, _scene())
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 16, 16)
    for mode in ("plain", "wavefront"):
        with pytest.raises(EosError) as e:
            api.render(ctx, dsc, cam, 1, spp=5, mode=mode, device=False, aa_grid=True)
        assert e.value.code == 1
    r = api.render(ctx, dsc, cam, 1, spp=4, device=False, aa_grid=True)
    assert r["rgb"].shape == (256, 3)


def test_aa_grid_backward_matches_fp64_adjoint(ctx):
    import torch
    sc = _scene()
    dsc = api.DeviceScene(ctx, sc)
    cams = [scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 40, 32)]
    td, spp = 2, 9
    r = api.render(ctx, dsc, cams[0], td, spp=spp, outputs=("rgb", "paths"), device=True, aa_grid=True)
    target = torch.rand(r["rgb"].shape, generator=torch.Generator(device="cuda").manual_seed(6), device="cuda") * 0.5
    g = 2.0 * (r["rgb"] - target)
    gm, gl = api.render_backward(ctx, dsc, cams, td, r["paths"], g.contiguous(), spp=spp, aa_grid=True)
    torch.cuda.synchronize()
    ph = r["paths"].cpu().numpy()
    mp = sc.materials.astype(np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    rgb64, gm64, gl64 = oracle.Oracle(sc).frozen_f64(cams, 40, 32, 0.5, td, ph[:, :8], ph[:, 8:].view(np.uint32), mp,
                                                     sc.lights.astype(np.float64),
                                                     g=g.cpu().numpy().astype(np.float64), spp=spp, aa_grid=True)
    r32 = r["rgb"].cpu().numpy()
    assert (np.abs(rgb64 - r32) / np.maximum(1.0, np.abs(rgb64))).max() < 1e-3
    for name, a, b in (("materials", gm.cpu().numpy(), gm64), ("lights", gl.cpu().numpy(), gl64)):
        err, scale = np.abs(a - b).max(), np.abs(b).max()
        assert err <= 1e-3 * max(scale, 1e-12), (name, err, scale)
