"""Stress workload (config 5): 4,524,288 triangles (800 instances of a 5,000-thin-triangle
cluster over a 512x512-cell height field), 8 lights, depth 4, 2 spp with jitter,
reflectivity up to 0.9."""
import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes
from tests.parity import RGB_TOL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stress(ctx):
    sc = scenes.config5_scene()
    return sc, api.DeviceScene(ctx, sc, inputs_on_device=True)


def test_stress_sampled_paths_match_oracle(ctx, stress):
    sc, dsc = stress
    assert sc.n_tris == 4_524_288
    cam = scenes.config5_camera(640, 360)
    g = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7, outputs=("rgb", "paths"),
                   device=True)
    pix = np.arange(0, cam.width * cam.height, 37, dtype=np.int32)
    o = oracle.Oracle(sc).render(cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7, pixels=pix)
    paths = g["paths"].cpu().numpy().reshape(-1, 2, 16)[pix].reshape(-1, 16)
    assert np.array_equal(paths[:, :8], o["hits"])
    assert np.array_equal(paths[:, 8:].view(np.uint32), o["shadows"])
    assert np.abs(g["rgb"].cpu().numpy()[pix] - o["rgb"]).max() <= RGB_TOL
    # thin triangles are rejected by |det| < 1e-5 like the reference: some rays pass them
    assert (o["hits"][:, 0] >= 0).mean() > 0.5


def test_stress_4k_wavefront_equals_plain(ctx, stress):
    sc, dsc = stress
    cam = scenes.config5_camera()
    a = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7, outputs=("rgb",), device=True)
    b = api.render(ctx, dsc, cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7, outputs=("rgb",), device=True,
                   mode="wavefront")
    assert bool((a["rgb"] == b["rgb"]).all())
    for k in ("primary_rays", "shadow_rays", "secondary_rays"):
        assert a["stats"][k] == b["stats"][k]
    assert a["stats"]["primary_rays"] == 3840 * 2160 * 2
