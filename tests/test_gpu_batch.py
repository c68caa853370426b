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
