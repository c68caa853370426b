"""Scene files (eos_scene_save / eos_scene_load): a loaded scene carries the same tree and
records as the one saved, so every render, batch and query of it equals the original's
bit for bit (gradients up to the order of their float atomics), and the loaded scene
alone still matches the oracle.  A missing, truncated, altered or foreign file is refused
with a status and leaves no scene behind.  Two builds of one scene save the same bytes."""
import ctypes

import numpy as np
import pytest

import oracle
from eos_b200 import _lib as L
from eos_b200 import api, scenes
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu

SAME_INFO = ("n_tris", "n_nodes", "leaf_size", "layout", "width", "builder", "depth", "sah_cost", "n_objects",
             "n_lights")


def _np(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else x


def _saved(ctx, tmp_path, sc, **build):
    dsc = api.DeviceScene(ctx, sc, **build)
    path = tmp_path / "scene.eos"
    dsc.save(path)
    return dsc, api.DeviceScene.load(ctx, path, sc), path


@pytest.mark.parametrize("build", [{}, {"builder": "lbvh"}, {"width": 2, "leaf_size": 1},
                                   {"layout": "fixed", "leaf_size": 4}])
def test_loaded_scene_renders_like_the_built_one(ctx, tmp_path, build):
    sc = scenes.small_random_scene(5, transparent=1, ambient_index=1.1)
    dsc, lsc, _ = _saved(ctx, tmp_path, sc, **build)
    a, b = dsc.info(), lsc.info()
    for k in SAME_INFO:
        assert a[k] == b[k], k
    assert b["build_ms"] == 0.0
    cam = scenes.look_at((1.0, 4.0, 9.0), (0, 0, 0), 50.0, 96, 72)
    for mode in ("plain", "wavefront"):
        outs = ("rgb", "rgba8", "hit", "paths") if mode == "plain" else ("rgb", "rgba8", "paths")
        ra = api.render(ctx, dsc, cam, 3, spp=2, jitter_seed=7, mode=mode, outputs=outs, device=False)
        rb = api.render(ctx, lsc, cam, 3, spp=2, jitter_seed=7, mode=mode, outputs=outs, device=False)
        for k in outs:
            assert np.array_equal(ra[k], rb[k]), (mode, k)
    o = oracle.Oracle(sc).render(cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7)
    p = _np(rb["paths"])
    assert np.array_equal(p[:, :8], o["hits"]) and np.array_equal(p[:, 8:].view(np.uint32), o["shadows"])
    assert np.abs(_np(rb["rgb"]) - o["rgb"]).max() <= RGB_TOL


@pytest.mark.parametrize("build", [{}, {"builder": "lbvh"}, {"width": 2, "leaf_size": 1}])
def test_builds_are_reproducible(ctx, tmp_path, build):
    """Two builds of one scene write the same file, byte for byte, but for the build time
    in the header (bytes 56..59): the records are numbered by scans, not by atomics."""
    sc = scenes.small_random_scene(11, n_spheres=40, level=4, lights=2)
    raw = []
    for k in range(2):
        d = api.DeviceScene(ctx, sc, **build)
        d.save(tmp_path / f"b{k}.eos")
        d.close()
        raw.append((tmp_path / f"b{k}.eos").read_bytes())
    assert len(raw[0]) == len(raw[1]) > 128 * 1000
    assert raw[0][:56] == raw[1][:56] and raw[0][60:] == raw[1][60:]


def test_loaded_scene_in_batches_queries_and_gradients(ctx, tmp_path):
    sc = scenes.small_random_scene(8, lights=3)
    dsc, lsc, _ = _saved(ctx, tmp_path, sc)
    cams = [scenes.look_at((x, 3.0, 8.0), (0, 0, 0), 55.0, 64, 48) for x in (-2.0, 0.5, 3.0)]
    jobs = [api.BatchJob(s, c, 2) for s in (dsc, lsc) for c in cams]
    outs = api.make_batch_outputs(jobs, outputs=("rgb", "paths"))
    api.render_batch(ctx, jobs, outs)
    for j in range(3):
        for k in ("rgb", "paths"):
            assert np.array_equal(_np(outs[j][k]), _np(outs[j + 3][k])), (j, k)
    rng = np.random.default_rng(1)
    rays = np.concatenate([rng.uniform(-3, 3, (4096, 3)), rng.normal(size=(4096, 3))], 1).astype(np.float32)
    rays[:, 3:] /= np.linalg.norm(rays[:, 3:], axis=1, keepdims=True)
    for fn in (api.trace_closest, api.trace_any):
        ra, rb = fn(ctx, dsc, rays), fn(ctx, lsc, rays)
        for x, y in zip(ra if isinstance(ra, tuple) else (ra,), rb if isinstance(rb, tuple) else (rb,)):
            assert np.array_equal(_np(x), _np(y)), fn.__name__
    r = api.render(ctx, dsc, cams[1], 2, outputs=("rgb", "paths"), device=True)
    d_rgb = np.random.default_rng(2).normal(size=_np(r["rgb"]).shape).astype(np.float32)
    import torch
    d_rgb = torch.from_numpy(d_rgb).cuda()
    ga = api.render_backward(ctx, dsc, [cams[1]], 2, r["paths"], d_rgb)
    gb = api.render_backward(ctx, lsc, [cams[1]], 2, r["paths"], d_rgb)
    for x, y in zip(ga, gb):  # the adjoint sums with float atomics: equal up to their order
        assert (x - y).abs().max() <= 1e-5 * x.abs().max()


def test_edge_and_multi_chunk_scenes(ctx, tmp_path):
    """Empty, one- and two-triangle scenes (single root record), and a 205k-triangle scene
    whose payload spans several staging chunks with part boundaries inside them."""
    mat = np.array([[0.5, 0.5, 0.5, 0.2, 0.2, 0.2, 16, 0.3]], np.float32)
    light = np.array([[2, 2, 2, 1, 1, 1]], np.float32)
    V = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0], [0, 0, 1], [0, 0, 1], [0, 0, 1]], np.float32)
    N = np.tile([[0, 0, 1]], (6, 1)).astype(np.float32)
    cases = [scenes.SceneData(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), mat, light)]
    for tris in (np.array([[0, 1, 2]]), np.array([[0, 1, 2], [3, 4, 5]])):
        cases.append(scenes.SceneData(V, N, tris, np.zeros(len(tris)), mat, light))
    cases.append(scenes.small_random_scene(11, n_spheres=10, level=5))
    assert cases[-1].n_tris > 200_000
    for i, sc in enumerate(cases):
        dsc, lsc, path = _saved(ctx, tmp_path, sc)
        if i == 3:
            assert path.stat().st_size > 2 * 8 * 2**20
        cam = scenes.look_at((0.5, 1.0, 5.0), (0, 0, 0), 60, 80, 48)
        ra = api.render(ctx, dsc, cam, 2, outputs=("rgb", "paths"), device=False)
        rb = api.render(ctx, lsc, cam, 2, outputs=("rgb", "paths"), device=False)
        assert np.array_equal(ra["rgb"], rb["rgb"]) and np.array_equal(ra["paths"], rb["paths"]), i
        if sc.n_tris:
            assert np.array_equal(dsc.morton()[1], lsc.morton()[1]), i
        lsc.close()
        dsc.close()


def test_material_and_light_edits_after_load(ctx, tmp_path):
    sc = scenes.small_random_scene(9)
    dsc, lsc, _ = _saved(ctx, tmp_path, sc)
    mats = np.asarray(scenes.pad_materials(sc.materials)).copy()
    mats[:, 0] *= 0.5
    lights = np.asarray(sc.lights, np.float32).copy()
    lights[0, :3] += 1.0
    for s in (dsc, lsc):
        s.set_materials(mats)
        s.set_lights(lights)
    cam = scenes.look_at((0.0, 5.0, 7.0), (0, 0, 0), 50.0, 64, 64)
    ra = api.render(ctx, dsc, cam, 2, outputs=("rgb",), device=False)
    rb = api.render(ctx, lsc, cam, 2, outputs=("rgb",), device=False)
    assert np.array_equal(ra["rgb"], rb["rgb"])


def test_scene_file_errors(ctx, tmp_path):
    sc = scenes.small_random_scene(2)
    dsc, _, path = _saved(ctx, tmp_path, sc)
    raw = path.read_bytes()
    lib = ctx.lib

    def load_status(data):
        p = tmp_path / "bad.eos"
        p.write_bytes(data)
        h = ctypes.c_void_p()
        code = lib.eos_scene_load(ctx.h, str(p).encode(), ctypes.byref(h))
        assert not h.value
        return code

    h = ctypes.c_void_p()
    assert lib.eos_scene_load(ctx.h, str(path).encode(), ctypes.byref(h)) == 0
    assert lib.eos_scene_destroy(h) == 0
    assert load_status(raw[: len(raw) - 1]) == 10          # truncated payload
    assert load_status(raw[:50]) == 10                      # truncated header
    assert load_status(b"") == 10
    flipped = bytearray(raw)
    flipped[-100] ^= 0x10
    assert load_status(bytes(flipped)) == 10                # checksum
    magic = bytearray(raw)
    magic[0:8] = b"NOTSCENE"
    assert load_status(bytes(magic)) == 10
    sizes = bytearray(raw)
    sizes[16] ^= 0x01                                       # n_nodes no longer matches the payload
    assert load_status(bytes(sizes)) == 10
    h = ctypes.c_void_p()
    assert lib.eos_scene_load(ctx.h, str(tmp_path / "missing.eos").encode(), ctypes.byref(h)) == 9
    assert lib.eos_scene_save(dsc.h, str(tmp_path / "no_such_dir" / "x.eos").encode()) == 9
    assert lib.eos_scene_save(None, str(path).encode()) == 1
    assert lib.eos_scene_load(None, str(path).encode(), ctypes.byref(h)) == 1
    d = scenes.instanced_test_scene(3, n_instances=2, lights=1)
    meshes = [api.DeviceScene(ctx, m) for m in d.meshes]
    inst = api.InstancedScene(ctx, meshes, d.instances, d.materials, d.lights)
    with pytest.raises(L.EosError) as e:
        inst.save(tmp_path / "inst.eos")
    assert e.value.code == 7
