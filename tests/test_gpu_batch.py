"""Batching (config-3 shape): many views of resident scenes with uneven resolution and
triangle count through one eos_render_batch call, replayed as a CUDA graph; every job
equals its own plain render bit for bit, and sampled paths equal the oracle."""
import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes

pytestmark = pytest.mark.gpu


def test_config3_style_batch_matches_plain_and_oracle(ctx):
    import torch
    jobs_spec = scenes.config3_jobs(n_views=10, n_scenes=3, tri_range=(10_000, 60_000))
    dev_scenes = {}
    jobs = []
    for j in jobs_spec:
        key = id(j.scene)
        if key not in dev_scenes:
            dev_scenes[key] = api.DeviceScene(ctx, j.scene)
        jobs.append(api.BatchJob(dev_scenes[key], j.camera, j.trace_depth, j.pixel_offset))
    assert len({id(j.scene) for j in jobs_spec}) == 4
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"))
    st = None
    for _ in range(2):  # capture, then replay
        st = api.render_batch(ctx, jobs, outs)
    torch.cuda.synchronize()
    assert st["primary_rays"] == sum(j.camera.width * j.camera.height for j in jobs)
    rng = np.random.default_rng(5)
    for spec, j, o in zip(jobs_spec, jobs, outs):
        ref = api.render(ctx, j.scene, j.camera, j.trace_depth, j.pixel_offset, outputs=("rgb", "paths"),
                         device=False)
        assert np.array_equal(o["rgb"].cpu().numpy(), ref["rgb"])
        assert np.array_equal(o["paths"].cpu().numpy(), ref["paths"])
    # sampled paths of two jobs against the oracle
    for spec, o in list(zip(jobs_spec, outs))[::6]:
        npx = spec.camera.width * spec.camera.height
        pix = np.sort(rng.choice(npx, min(npx, 3000), replace=False)).astype(np.int32)
        r = oracle.Oracle(spec.scene).render(spec.camera, spec.trace_depth, pixel_offset=spec.pixel_offset,
                                             pixels=pix)
        p = o["paths"].cpu().numpy()[pix]
        assert np.array_equal(p[:, :8], r["hits"])
        assert np.array_equal(p[:, 8:].view(np.uint32), r["shadows"])


def test_async_batches_equal_synchronous_ones(ctx):
    """EOS_FLAG_ASYNC: three batches in a row into pinned host images (each call's copy to
    the host overlaps the next call's rendering) give the synchronous call's images and
    stats once the context is synchronized; a device error of an asynchronous call is
    reported by the synchronize, and the context stays usable."""
    import torch
    from eos_b200._lib import EosError
    sc = scenes.small_random_scene(41, n_spheres=6, level=3, lights=3, refl=0.6)
    dsc = api.DeviceScene(ctx, sc)
    cams = [scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 160, 120),
            scenes.look_at((-6.0, 4.0, 6.0), (0, -0.5, 0), 50.0, 96, 64),
            scenes.look_at((3.0, 2.0, 7.0), (0, -0.5, 0), 55.0, 1280, 960)]  # the pass runs as two lanes
    jobs = [api.BatchJob(dsc, c, 2, 0.5) for c in cams]
    ref_outs = [{"rgba8": np.zeros((c.height, c.width, 4), np.uint8)} for c in cams]
    ref_st = api.render_batch(ctx, jobs, ref_outs)
    host = [[{"rgba8": torch.zeros((c.height, c.width, 4), dtype=torch.uint8).pin_memory()} for c in cams]
            for _ in range(3)]
    for outs in host:
        assert api.render_batch(ctx, jobs, [{"rgba8": o["rgba8"].numpy()} for o in outs], async_outputs=True) is None
    stats = ctx.synchronize()
    assert len(stats) == 3
    for outs, st in zip(host, stats):
        for o, r in zip(outs, ref_outs):
            assert np.array_equal(o["rgba8"].numpy(), r["rgba8"])
        for k in ("primary_rays", "shadow_rays", "secondary_rays"):
            assert st[k] == ref_st[k]
    # a device error of an asynchronous call surfaces at the synchronize
    ctx.set_limits(queue_entries=16)
    try:
        api.render_batch(ctx, jobs, [{"rgba8": o["rgba8"].numpy()} for o in host[0]], async_outputs=True)
        with pytest.raises(EosError) as e:
            ctx.synchronize()
        assert e.value.code == 6
    finally:
        ctx.set_limits()
    out = [{"rgba8": np.zeros((c.height, c.width, 4), np.uint8)} for c in cams]
    api.render_batch(ctx, jobs, out)
    assert all(np.array_equal(a["rgba8"], b["rgba8"]) for a, b in zip(out, ref_outs))


def test_batch_over_several_chunks_equals_single_renders(ctx):
    """A batch of more than 2^24 paths runs as two chunks, each with its bounces overlapped
    across streams: nine 1080p views (18.7M paths) equal nine single renders bit for bit,
    and a batch of two-sample jobs (the resolve pass) as well."""
    import torch
    sc = scenes.small_random_scene(41, n_spheres=6, level=3, lights=2, refl=0.6, transparent=1)
    dsc = api.DeviceScene(ctx, sc)
    cams = [scenes.look_at((4.0 * np.cos(a), 2.5, 4.0 * np.sin(a) + 4.0), (0, -0.5, 0), 55.0, 1920, 1080)
            for a in np.linspace(0.2, 2.9, 9)]
    jobs = [api.BatchJob(dsc, c, 2, 0.5) for c in cams]
    assert sum(c.width * c.height for c in cams) > 1 << 24
    outs = api.make_batch_outputs(jobs, ("rgb",))
    for _ in range(2):  # capture, then replay
        st = api.render_batch(ctx, jobs, outs)
    torch.cuda.synchronize()
    assert st["primary_rays"] == 9 * 1920 * 1080 and st["secondary_rays"] > 0
    for c, o in zip(cams, outs):
        ref = api.render(ctx, dsc, c, 2, 0.5, outputs=("rgb",), device=True)
        assert torch.equal(o["rgb"], ref["rgb"])
    small = [scenes.look_at((1.0, 2.5, 8.0 - k), (0, -0.5, 0), 55.0, 160, 120) for k in range(3)]
    jobs2 = [api.BatchJob(dsc, c, 2, 0.5, 2, 11) for c in small]
    outs2 = api.make_batch_outputs(jobs2, ("rgb", "paths"))
    api.render_batch(ctx, jobs2, outs2)
    for c, o in zip(small, outs2):
        ref = api.render(ctx, dsc, c, 2, 0.5, spp=2, jitter_seed=11, outputs=("rgb", "paths"), device=False)
        assert np.array_equal(o["rgb"].cpu().numpy(), ref["rgb"])
        assert np.array_equal(o["paths"].cpu().numpy(), ref["paths"])


def test_batching_workload_matches_reference_goldens(ctx):
    """Jobs of the batching workload (scenes.config3_jobs: 8 views of the config-1 scene and
    its 16 mixed scenes, one batch): the reference's own renderer recorded 20,000 sampled
    paths of job 69 (its largest mixed scene) and of job 0 (a 1080p view of the config-1
    scene), and 2,000 of each of the other 15 mixed scenes -- the batch equals them on every
    path but the classes the oracle flags, and equals the oracle everywhere."""
    import os
    from tests.parity import RGB_TOL, classify, path_mismatch
    golden = os.path.join(os.path.dirname(__file__), "golden")
    if not all(os.path.exists(os.path.join(golden, f"config3_job{k}.npz")) for k in (0, 69)):
        pytest.skip("config3 goldens not generated")
    spec = scenes.config3_jobs()
    keep = list(range(8)) + [k for k, j in enumerate(spec) if j.scene.name.startswith("mixed")]
    dev = {}
    jobs = []
    for k in keep:
        j = spec[k]
        if id(j.scene) not in dev:
            dev[id(j.scene)] = api.DeviceScene(ctx, j.scene)
        jobs.append(api.BatchJob(dev[id(j.scene)], j.camera, j.trace_depth, j.pixel_offset))
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"))
    api.render_batch(ctx, jobs, outs)
    for k in (0, 69):
        gd = np.load(os.path.join(golden, f"config3_job{k}.npz"))
        pix = gd["pixels"]
        o_k = outs[keep.index(k)]
        p = o_k["paths"].cpu().numpy()[pix]
        gh, gs = p[:, :8], p[:, 8:].view(np.uint32)
        j = spec[k]
        o = oracle.Oracle(j.scene).render(j.camera, j.trace_depth, pixel_offset=j.pixel_offset, pixels=pix)
        mm = path_mismatch(gh, gs, gd["hits"], gd["shadows"], j.trace_depth + 1)
        c = classify(mm, o["flags"])
        print(f"config3 job {k} vs reference:", c)
        assert c["unexplained"] == 0, c
        assert c["axis_parallel_not_tie"] + c["near_origin_not_tie"] <= 10, c
        assert np.abs(o_k["rgb"].cpu().numpy()[pix] - gd["rgb"]).max(1)[~mm].max() <= RGB_TOL
        assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"])
        ref = api.render(ctx, jobs[keep.index(k)].scene, j.camera, j.trace_depth, j.pixel_offset,
                         outputs=("rgb", "paths"), device=False)
        assert np.array_equal(o_k["paths"].cpu().numpy(), ref["paths"])
    # the other 15 mixed scenes: 2,000 sampled paths of each from the reference's renderer
    gm = np.load(os.path.join(golden, "config3_mixed.npz"))
    for k in np.unique(gm["job"]):
        k = int(k)
        sel = gm["job"] == k
        pix = gm["pixels"][sel]
        o_k = outs[keep.index(k)]
        p = o_k["paths"].cpu().numpy()[pix]
        gh, gs = p[:, :8], p[:, 8:].view(np.uint32)
        j = spec[k]
        o = oracle.Oracle(j.scene).render(j.camera, j.trace_depth, pixel_offset=j.pixel_offset, pixels=pix)
        mm = path_mismatch(gh, gs, gm["hits"][sel], gm["shadows"][sel], j.trace_depth + 1)
        c = classify(mm, o["flags"])
        assert c["unexplained"] == 0, (k, c)
        assert c["axis_parallel_not_tie"] + c["near_origin_not_tie"] <= 5, (k, c)
        assert np.abs(o_k["rgb"].cpu().numpy()[pix] - gm["rgb"][sel]).max(1)[~mm].max() <= RGB_TOL, k
        assert np.array_equal(gh, o["hits"]) and np.array_equal(gs, o["shadows"]), k
