"""Two-level scenes (eos_scene_create_instanced): the GPU traversal with rays moved into
each instance's object space equals the oracle's restatement (every instance tested, no
instance tree) bit for bit on hit ids and paths, in plain and batched mode; queries,
mixed batches, the 4.5M-triangle config-5 scene as 801 instances, and the errors."""
import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu


def _paths(p):
    p = p.cpu().numpy() if hasattr(p, "cpu") else p
    return p[:, :8], p[:, 8:].view(np.uint32)


def _device(ctx, d):
    meshes = [api.DeviceScene(ctx, m) for m in d.meshes]
    return api.InstancedScene(ctx, meshes, d.instances, d.materials, d.lights, d.ambient_index)


@pytest.mark.parametrize("seed,transparent,spp", [(3, 0, 1), (4, 2, 2)])
def test_instanced_scene_matches_oracle(ctx, seed, transparent, spp):
    d = scenes.instanced_test_scene(seed, n_instances=12, lights=2, transparent=transparent)
    dsc = _device(ctx, d)
    info = dsc.info()
    assert info["n_tris"] == d.n_tris
    cam = scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 120, 90)
    o = oracle.OracleInstanced(d).render(cam, 3, pixel_offset=0.5, spp=spp, jitter_seed=2)
    for mode in ("plain", "wavefront"):
        g = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, spp=spp, jitter_seed=2, mode=mode,
                       outputs=("rgb", "paths"), device=False)
        gh, gs = _paths(g["paths"])
        assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"]), mode
        assert np.abs(g["rgb"] - o["rgb"]).max() <= RGB_TOL, mode
    assert (o["hits"][:, 0] >= 0).mean() > 0.2


def test_instanced_queries_match_oracle(ctx):
    d = scenes.instanced_test_scene(5, n_instances=16)
    dsc = _device(ctx, d)
    rng = np.random.default_rng(6)
    rays = np.concatenate([rng.uniform(-4, 4, (20000, 3)), rng.normal(size=(20000, 3))], 1).astype(np.float32)
    rays[:, 3:] /= np.linalg.norm(rays[:, 3:], axis=1, keepdims=True)
    orc = oracle.OracleInstanced(d)
    ids, t = api.trace_closest(ctx, dsc, rays)
    oid, ot, _ = orc.closest(rays)
    assert np.array_equal(ids, oid)
    assert np.array_equal(t[ids >= 0], ot[oid >= 0])
    assert np.array_equal(api.trace_any(ctx, dsc, rays), orc.any(rays))
    assert (ids >= 0).mean() > 0.05


def test_identity_instances_equal_the_flat_scene(ctx):
    """One instance with the identity transform renders exactly as the mesh itself."""
    sc = scenes.small_random_scene(21, n_spheres=5, level=2, lights=2, refl=0.5)
    flat = api.DeviceScene(ctx, sc)
    d = scenes.InstancedData([sc], [(0, np.hstack([np.eye(3), np.zeros((3, 1))]), 0)], sc.materials, sc.lights)
    inst = _device(ctx, d)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 96, 72)
    a = api.render(ctx, flat, cam, 3, outputs=("rgb", "paths"), device=False)
    b = api.render(ctx, inst, cam, 3, outputs=("rgb", "paths"), device=False)
    assert np.array_equal(a["paths"], b["paths"])
    assert np.abs(a["rgb"] - b["rgb"]).max() <= RGB_TOL


def test_mixed_batch_of_flat_and_instanced_scenes(ctx):
    import torch
    d = scenes.instanced_test_scene(7)
    inst = _device(ctx, d)
    flat = api.DeviceScene(ctx, scenes.small_random_scene(22, n_spheres=4, level=2, lights=2))
    jobs = [api.BatchJob(inst, scenes.look_at((1, 3, 9), (0, 0, 0), 50, 128, 96), 2),
            api.BatchJob(flat, scenes.look_at((0, 3, 8), (0, 0, 0), 50, 96, 64), 2),
            api.BatchJob(inst, scenes.look_at((-6, 2, 4), (0, 0, 0), 60, 64, 64), 3, spp=2, jitter_seed=1)]
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"))
    api.render_batch(ctx, jobs, outs)
    torch.cuda.synchronize()
    for j, o in zip(jobs, outs):
        ref = api.render(ctx, j.scene, j.camera, j.trace_depth, j.pixel_offset, spp=j.spp, jitter_seed=j.jitter_seed,
                         outputs=("rgb", "paths"), device=False)
        assert np.array_equal(o["paths"].cpu().numpy(), ref["paths"])
        assert np.array_equal(o["rgb"].cpu().numpy(), ref["rgb"])


def test_config5_as_instances_matches_oracle_on_sampled_pixels(ctx):
    """801 instances (the height field and the 5,000-triangle cluster 800 times) at 4K:
    sampled pixels against the oracle; the mesh is stored once."""
    d = scenes.config5_instanced()
    dsc = _device(ctx, d)
    flat_bytes = 96 * d.n_tris  # triangle + shading records of the flattened scene alone
    assert dsc.info()["device_bytes"] + sum(m.info()["device_bytes"] for m in dsc.meshes) < flat_bytes
    cam = scenes.config5_camera()
    rng = np.random.default_rng(8)
    pix = rng.choice(cam.width * cam.height, 192, replace=False).astype(np.int32)
    o = oracle.OracleInstanced(d).render(cam, 1, pixel_offset=0.5, pixels=pix)
    g = api.render(ctx, dsc, cam, 1, pixel_offset=0.5, mode="wavefront", outputs=("rgb", "paths"), device=False)
    gh, gs = _paths(g["paths"])
    assert np.array_equal(gh[pix], o["hits"]) and np.array_equal(gs[pix], o["shadows"])
    assert np.abs(g["rgb"][pix] - o["rgb"]).max() <= RGB_TOL
    assert (o["hits"][:, 0] >= 0).mean() > 0.5


def test_instanced_errors(ctx):
    from eos_b200._lib import EosError
    d = scenes.instanced_test_scene(9, n_instances=3)
    meshes = [api.DeviceScene(ctx, m) for m in d.meshes]
    bad = list(d.instances)
    bad[1] = (bad[1][0], np.zeros((3, 4)), bad[1][2])  # singular transform
    with pytest.raises(EosError) as e:
        api.InstancedScene(ctx, meshes, bad, d.materials, d.lights)
    assert e.value.code == 1
    with pytest.raises(EosError):  # material base beyond the table
        api.InstancedScene(ctx, meshes, [(0, d.instances[0][1], 99)], d.materials, d.lights)
    inst = api.InstancedScene(ctx, meshes, d.instances, d.materials, d.lights)
    with pytest.raises(EosError) as e:  # scene files hold flat scenes only
        inst.save("/nonexistent-dir/never-written.eosscn")
    assert e.value.code == 7


@pytest.mark.parametrize("spp", [1, 2])
def test_instanced_backward_matches_fp64_adjoint(ctx, spp):
    """The adjoint of a two-level scene (each recorded hit replayed in its instance's object
    space) against the oracle's FP64 adjoint of the same frozen paths, within 1e-3 relative."""
    import torch
    d = scenes.instanced_test_scene(7, n_instances=10, lights=2, transparent=1)
    d.materials[1:, 7] = np.where(d.materials[1:, 8] > 0, 0.0, 0.3)
    dsc = _device(ctx, d)
    cams = [scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 48, 40),
            scenes.look_at((-6.0, 4.0, 5.0), (0, -0.5, 0), 55.0, 48, 40)]
    td = 2
    paths, rgb = [], []
    for c in cams:
        r = api.render(ctx, dsc, c, td, pixel_offset=0.5, spp=spp, jitter_seed=3, outputs=("rgb", "paths"), device=True)
        paths.append(r["paths"])
        rgb.append(r["rgb"])
    paths = torch.cat(paths)
    rgb = torch.cat(rgb)
    target = torch.from_numpy(np.random.default_rng(6).uniform(0, 0.6, tuple(rgb.shape)).astype(np.float32)).cuda()
    g = 2.0 * (rgb - target)
    gm, gl = api.render_backward(ctx, dsc, cams, td, paths, g, pixel_offset=0.5, spp=spp, jitter_seed=3)
    mp = np.asarray(d.materials, np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    lp = np.asarray(d.lights, np.float64)
    p = paths.cpu().numpy()
    rgb64, om, ol = oracle.OracleInstanced(d).frozen_f64(cams, 48, 40, 0.5, td, p[:, :8], p[:, 8:].view(np.uint32),
                                                         mp, lp, g=g.cpu().numpy().astype(np.float64), spp=spp,
                                                         jitter_seed=3)
    r32 = rgb.cpu().numpy()
    assert (np.abs(rgb64 - r32) / np.maximum(1.0, np.abs(rgb64))).max() < 1e-3
    gm, gl = gm.cpu().numpy(), gl.cpu().numpy()
    for name, a, b in [("materials", gm, om), ("lights", gl, ol)]:
        err, scale = np.abs(a - b).max(), np.abs(b).max()
        assert err <= 1e-3 * max(scale, 1e-12), (name, err, scale)
