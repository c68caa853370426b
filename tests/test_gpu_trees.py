"""Materials that are both reflective and transparent: the reference traces the mirror ray
and then the transparent bounce's ray from the same hit (src/RayTracer.cpp:339-407), so a
path is a binary tree of rays.  The GPU renders it in plain and batched mode with tree-form
records (EOS_FLAG_TREE_RECORDS, heap order), against the reference's own output (golden
both91.npz) and the oracle, and differentiates it against the FP64 tree adjoint."""
import os

import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes
from eos_b200._lib import EosError
from tests.parity import RGB_TOL, classify

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
UNSUPPORTED = 7


def tree_scene():
    return scenes.small_random_scene(91, n_spheres=7, level=2, lights=3, refl=0.5, transparent=1, both=3,
                                     ambient_index=1.0002)


def split(p):
    p = p.cpu().numpy() if hasattr(p, "cpu") else p
    return p[..., 0], p[..., 1].view(np.uint32)


@pytest.mark.parametrize("mode", ["plain", "wavefront", "batch"])
def test_trees_match_reference_golden(ctx, mode):
    gd = np.load(os.path.join(GOLDEN, "both91.npz"))
    W, H, td = (int(v) for v in gd["size"])
    cam = scenes.CameraData(*[gd["cam"][3 * i:3 * i + 3] for i in range(4)], W, H)
    sc = tree_scene()
    dsc = api.DeviceScene(ctx, sc)
    if mode == "batch":
        jobs = [api.BatchJob(dsc, cam, td, 0.0)]
        outs = api.make_batch_outputs(jobs, ("rgb", "paths"), tree_records=True)
        st = api.render_batch(ctx, jobs, outs, tree_records=True)
        rgb, paths = outs[0]["rgb"].cpu().numpy(), outs[0]["paths"]
    else:
        r = api.render(ctx, dsc, cam, td, pixel_offset=0.0, mode=mode, outputs=("rgb", "paths"), device=False,
                       tree_records=True)
        rgb, paths, st = r["rgb"], r["paths"], r["stats"]
    gh, gs = split(paths)
    assert gh.shape == (W * H, 15)
    o = oracle.Oracle(sc).render_tree(cam, td, pixel_offset=0.0)
    mm = (gh != gd["hits"]).any(1) | (gs != gd["shadows"]).any(1)
    c = classify(mm, o["flags"])
    assert c["unexplained"] == 0, c
    assert np.abs(rgb - gd["rgb"]).max(1)[~mm].max() <= RGB_TOL
    assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"])
    assert np.abs(rgb - o["rgb"]).max() <= RGB_TOL
    assert (st["primary_rays"], st["shadow_rays"], st["secondary_rays"]) == tuple(int(v) for v in gd["counts"])
    both = ((gh[:, 1:15:2] != -2) & (gh[:, 2:15:2] != -2)).any(1)
    assert both.sum() > 50  # paths that traced both rays of one hit


def test_trees_two_samples_and_modes_agree(ctx):
    """2 jittered samples per pixel, depth 5, ragged tiles: plain, wavefront and the batch
    (mixed with a chain scene) give the same tree records and colours, equal to the oracle."""
    sc = tree_scene()
    dsc = api.DeviceScene(ctx, sc)
    chain = api.DeviceScene(ctx, scenes.small_random_scene(31, n_spheres=4, level=2, lights=2, refl=0.6))
    cam = scenes.look_at((0.8, 2.0, 7.5), (0, -0.5, 0), 55.0, 61, 37)
    td = 4
    a = api.render(ctx, dsc, cam, td, spp=2, jitter_seed=9, outputs=("rgb", "paths", "hit"), device=False,
                   tree_records=True)
    b = api.render(ctx, dsc, cam, td, spp=2, jitter_seed=9, mode="wavefront", outputs=("rgb", "paths"),
                   device=False, tree_records=True)
    assert np.array_equal(a["paths"], b["paths"]) and np.array_equal(a["rgb"], b["rgb"])
    assert np.array_equal(a["hit"], a["paths"][:, 0, 0])
    jobs = [api.BatchJob(chain, cam, 2, 0.5), api.BatchJob(dsc, cam, td, 0.5, 2, 9)]
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"), tree_records=True)
    api.render_batch(ctx, jobs, outs, tree_records=True)
    assert np.array_equal(outs[1]["paths"].cpu().numpy(), a["paths"])
    assert np.array_equal(outs[1]["rgb"].cpu().numpy(), a["rgb"])
    o = oracle.Oracle(sc).render_tree(cam, td, pixel_offset=0.5, spp=2, jitter_seed=9)
    gh, gs = split(a["paths"])
    assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"])
    assert np.abs(a["rgb"] - o["rgb"]).max() <= RGB_TOL
    # the chain job of the same batch keeps its chain colours, its tree records hold the chain
    c = api.render(ctx, chain, cam, 2, outputs=("rgb", "paths"), device=False)
    assert np.array_equal(outs[0]["rgb"].cpu().numpy(), c["rgb"])
    th = outs[0]["paths"].cpu().numpy()[..., 0]
    assert np.array_equal(th[:, 0], c["paths"][:, 0])


def test_trees_in_a_pass_of_two_lanes(ctx):
    """A ray-tree view of more than 2^20 paths (halves side by side, the init and resolve
    passes of tree mode in each): tree records and colours equal the plain renderer's."""
    import torch
    dsc = api.DeviceScene(ctx, tree_scene())
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 1280, 960)
    jobs = [api.BatchJob(dsc, cam, 3, 0.5)]
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"), tree_records=True)
    api.render_batch(ctx, jobs, outs, tree_records=True)
    ref = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, outputs=("rgb", "paths"), device=True, tree_records=True)
    torch.cuda.synchronize()
    assert torch.equal(outs[0]["paths"], ref["paths"])
    assert torch.equal(outs[0]["rgb"], ref["rgb"])


def test_tree_kernels_equal_chain_kernels_on_chain_scenes(ctx):
    """Tree records on a scene without such materials: the ray-tree kernels give the chain
    kernels' colours bit for bit and the chain bounces at their nodes."""
    sc = scenes.small_random_scene(11, n_spheres=5, level=2, lights=3, refl=0.6, transparent=2)
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 96, 72)
    for mode in ("plain", "wavefront"):
        a = api.render(ctx, dsc, cam, 3, mode=mode, outputs=("rgb", "paths"), device=False)
        b = api.render(ctx, dsc, cam, 3, mode=mode, outputs=("rgb", "paths"), device=False, tree_records=True)
        assert np.array_equal(a["rgb"], b["rgb"])
        for k in ("primary_rays", "shadow_rays", "secondary_rays"):
            assert a["stats"][k] == b["stats"][k]
        assert np.array_equal(b["paths"][:, 0, 0], a["paths"][:, 0])


def test_chain_records_of_a_tree_scene_are_refused(ctx):
    sc = tree_scene()
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 32, 24)
    for mode in ("plain", "wavefront"):
        with pytest.raises(EosError) as e:
            api.render(ctx, dsc, cam, 2, mode=mode, outputs=("rgb", "paths"), device=False)
        assert e.value.code == UNSUPPORTED
        r = api.render(ctx, dsc, cam, 2, mode=mode, outputs=("rgb",), device=False)  # colours alone are fine
        assert r["rgb"].shape == (32 * 24, 3)
    with pytest.raises(EosError) as e:
        api.render_backward(ctx, dsc, [cam], 2, np.zeros((32 * 24, 16), np.int32), np.zeros((32 * 24, 3), np.float32),
                            device=False)
    assert e.value.code == UNSUPPORTED


@pytest.mark.parametrize("spp", [1, 2])
def test_tree_backward_matches_fp64_adjoint(ctx, spp):
    """The GPU adjoint over ray trees (visibility frozen from the tree records) against the
    oracle's FP64 tree adjoint, within 1e-3 relative."""
    import torch
    sc = tree_scene()
    dsc = api.DeviceScene(ctx, sc)
    cams = [scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 48, 40),
            scenes.look_at((-5.0, 3.0, 6.0), (0, -0.5, 0), 55.0, 48, 40)]
    td = 3
    paths, rgbs = [], []
    for c in cams:
        r = api.render(ctx, dsc, c, td, spp=spp, jitter_seed=3, outputs=("rgb", "paths"), device=True,
                       tree_records=True)
        paths.append(r["paths"])
        rgbs.append(r["rgb"])
    paths = torch.cat(paths)
    rgb = torch.cat(rgbs)
    target = torch.rand(rgb.shape, generator=torch.Generator(device="cuda").manual_seed(5), device="cuda") * 0.5
    g = 2.0 * (rgb - target)
    gm, gl = api.render_backward(ctx, dsc, cams, td, paths, g.contiguous(), spp=spp, jitter_seed=3,
                                 tree_records=True)
    torch.cuda.synchronize()
    ph = paths.cpu().numpy()
    mp = sc.materials.astype(np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    rgb64, gm64, gl64 = oracle.Oracle(sc).frozen_f64(cams, 48, 40, 0.5, td, ph[..., 0], ph[..., 1].view(np.uint32),
                                                     mp, sc.lights.astype(np.float64),
                                                     g=g.cpu().numpy().astype(np.float64), spp=spp, jitter_seed=3,
                                                     tree=True)
    r32 = rgb.cpu().numpy()
    assert (np.abs(rgb64 - r32) / np.maximum(1.0, np.abs(rgb64))).max() < 1e-3
    for name, a, b in (("materials", gm.cpu().numpy(), gm64), ("lights", gl.cpu().numpy(), gl64)):
        err, scale = np.abs(a - b).max(), np.abs(b).max()
        assert err <= 1e-3 * max(scale, 1e-12), (name, err, scale)
    assert np.abs(gm64[1:4]).sum() > 0  # the both-material objects take gradient


def test_noalloc_refuses_trees(ctx):
    import ctypes
    from ctypes import byref
    import torch
    from eos_b200 import _lib as L
    dsc = api.DeviceScene(ctx, tree_scene())
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 32, 24)
    rgb = torch.zeros((32 * 24, 3), device="cuda")
    c = api.camera_struct(cam)
    p = api.params_struct(2, 0.5, 1)
    code = ctx.lib.eos_render_noalloc(dsc.h, byref(c), byref(p), None, ctypes.c_void_p(rgb.data_ptr()), None,
                                      byref(L.Stats()))
    assert code == UNSUPPORTED
