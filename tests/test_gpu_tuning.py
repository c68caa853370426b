"""Tuning parameters change speed only: every block size / stack depth / queue chunk /
leaf size gives bit-identical images and paths; the autotuner writes and applies a table."""
import json

import numpy as np
import pytest

from eos_b200 import api, autotune, scenes

pytestmark = pytest.mark.gpu


def test_results_invariant_under_tuning(ctx):
    sc = scenes.small_random_scene(81, n_spheres=10, level=3, lights=3, refl=0.5)
    cam = scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 200, 150)
    ref = None
    for builder, layout, leaf, width in (("lbvh", "fixed", 1, 2), ("lbvh", "fixed", 3, 2), ("lbvh", "sah", 8, 2),
                                         ("lbvh", "sah", 32, 2), ("lbvh", "fixed", 32, 2), ("lbvh", "fixed", 1, 4),
                                         ("lbvh", "sah", 8, 4), ("lbvh", "fixed", 16, 4), ("ploc", "fixed", 1, 2),
                                         ("ploc", "sah", 8, 4), ("ploc", "fixed", 4, 4), ("ploc", "fixed", 32, 4)):
        dsc = api.DeviceScene(ctx, sc, leaf_size=leaf, layout=layout, width=width, builder=builder)
        assert dsc.info()["leaf_size"] == leaf and dsc.info()["width"] == width
        assert dsc.info()["builder"] == {"lbvh": 1, "ploc": 2}[builder]
        assert dsc.info()["sah_cost"] > 0
        for mode in ("plain", "wavefront"):
            for block, stack, chunk in ((64, 8, 32), (128, 16, 64), (256, 32, 256)):
                r = api.render(ctx, dsc, cam, 2, pixel_offset=0.5, mode=mode, outputs=("rgb", "paths"),
                               device=False, block_size=block, stack_depth=stack, queue_chunk=chunk)
                if ref is None:
                    ref = r
                    continue
                assert np.array_equal(r["paths"], ref["paths"]), (leaf, mode, block, stack, chunk)
                assert np.array_equal(r["rgb"], ref["rgb"]), (leaf, mode, block, stack, chunk)


def test_autotuner_writes_and_applies_table(ctx, tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "CANDIDATES", {"builder": ["ploc", "lbvh"], "width": [2, 4],
                                                 "layout": ["sah", "fixed"], "leaf_size": [2, 4],
                                                 "block_size": [64, 128], "stack_depth": [8, 16],
                                                 "queue_chunk": [64, 128]})
    sc = scenes.small_random_scene(82, n_spheres=12, level=3, lights=2)
    cams = [scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 160, 120)]
    path = tmp_path / "tuning.json"
    table = autotune.tune(ctx, [(sc, cams)], path=str(path), trace_depth=1, log=None)
    b = autotune.bucket_of(sc.n_tris)
    assert b in table and table[b]["mrays"] > 0
    saved = json.load(open(path))
    assert str(b) in saved["buckets"]
    # a scene created without build parameters now takes the tuned leaf size
    dsc = api.DeviceScene(ctx, sc, leaf_size=0)
    assert dsc.info()["leaf_size"] == table[b]["setting"]["leaf_size"]
    ctx.lib.eos_ctx_clear_tuning(ctx.h)
    info = api.DeviceScene(ctx, sc, leaf_size=0).info()
    assert info["leaf_size"] == 8 and info["layout"] == 1 and info["width"] == 4 and info["builder"] == 2
