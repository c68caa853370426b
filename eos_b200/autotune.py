"""Autotuner: hierarchy builder, node width / layout / leaf size, block size, queue chunk
and stack depth per scene-size bucket for the batched wavefront renderer.

For each bucket (triangle count rounded down to a power of two) the tuner renders a
representative job with coordinate descent over the candidate values: the tree parameters
first (builder, width, layout, leaf size: each change rebuilds the scene), then block size,
shared stack depth and queue chunk, keeping a value only when it is faster by more than the
noise margin.  The table is saved as JSON and registered with the library (eos_ctx_set_tuning), so render
calls that leave a parameter at 0 use the tuned value for their scene's bucket.
"""
from __future__ import annotations

import json
import math
import os
import time
from ctypes import byref

from . import _lib as L
from . import api

CANDIDATES = {
    "builder": ["ploc", "lbvh"],
    "width": [2, 4],
    "layout": ["sah", "fixed"],
    "leaf_size": [2, 4, 8, 16],
    "block_size": [64, 128, 256],
    "stack_depth": [8, 16, 32],
    "queue_chunk": [32, 64, 128],
}
DEFAULT = {"builder": "ploc", "width": 4, "layout": "fixed", "leaf_size": 4, "block_size": 128, "stack_depth": 16,
           "queue_chunk": 32}
LAYOUT_CODE = {"sah": L.LAYOUT_SAH, "fixed": L.LAYOUT_FIXED}
BUILDER_CODE = {"lbvh": L.BUILDER_LBVH, "ploc": L.BUILDER_PLOC}


def bucket_of(n_tris: int) -> int:
    return 1 << max(0, int(math.floor(math.log2(max(1, n_tris)))))


def _time_batch(ctx, jobs, outs, params, reps=3) -> float:
    import torch
    api.render_batch(ctx, jobs, outs, **params)  # warm-up (captures the graph)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        st = api.render_batch(ctx, jobs, outs, **params)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    rays = st["primary_rays"] + st["shadow_rays"] + st["secondary_rays"]
    return rays / (best * 1e-3) / 1e6  # Mrays/s


def tune_scene(ctx, scene_data, cameras, trace_depth=2, reps=3, margin=0.02, log=None, spp=1) -> dict:
    """Coordinate descent for one scene (its views rendered with `spp` jittered samples
    per pixel); returns the best setting and its Mrays/s."""
    best = dict(DEFAULT)
    scenes_by_leaf = {}

    def scene_for(builder, width, layout, leaf):
        key = (builder, width, layout, leaf)
        if key not in scenes_by_leaf:
            scenes_by_leaf[key] = api.DeviceScene(ctx, scene_data, leaf_size=leaf, inputs_on_device=True,
                                                  layout=layout, width=width, builder=builder)
        return scenes_by_leaf[key]

    def measure(setting):
        dsc = scene_for(setting["builder"], setting["width"], setting["layout"], setting["leaf_size"])
        jobs = [api.BatchJob(dsc, c, trace_depth, 0.5, spp, 7) for c in cameras]
        outs = api.make_batch_outputs(jobs, ("rgba8",))
        p = {k: setting[k] for k in ("block_size", "stack_depth", "queue_chunk")}
        return _time_batch(ctx, jobs, outs, p, reps)

    best_v = measure(best)
    trials = [(dict(best), best_v)]
    for key in ("builder", "width", "layout", "leaf_size", "block_size", "stack_depth", "queue_chunk"):
        for v in CANDIDATES[key]:
            if v == best[key]:
                continue
            cand = dict(best)
            cand[key] = v
            mv = measure(cand)
            trials.append((cand, mv))
            if log:
                log(f"  {cand} -> {mv:.1f} Mrays/s")
            if mv > best_v * (1 + margin):
                best, best_v = cand, mv
    for s in scenes_by_leaf.values():
        s.close()
    return {"setting": best, "mrays": best_v, "default_mrays": trials[0][1], "n_tris": scene_data.n_tris,
            "trials": [{"setting": t, "mrays": round(m, 1)} for t, m in trials]}


def apply_table(ctx, table: dict) -> None:
    """Registers a tuning table {bucket: {"setting": {...}}} with the library context."""
    ctx.lib.eos_ctx_clear_tuning(ctx.h)
    for bucket, entry in table.items():
        s = entry["setting"] if "setting" in entry else entry
        t = L.Tuning()
        t.block_size = int(s["block_size"])
        t.queue_chunk = int(s["queue_chunk"])
        t.stack_depth = int(s["stack_depth"])
        t.leaf_size = int(s["leaf_size"])
        t.layout = LAYOUT_CODE.get(s.get("layout", "sah"), L.LAYOUT_SAH)
        t.width = int(s.get("width", 2))
        t.builder = BUILDER_CODE.get(s.get("builder", "lbvh"), L.BUILDER_LBVH)
        L.check(ctx.lib.eos_ctx_set_tuning(ctx.h, int(bucket), byref(t)), "eos_ctx_set_tuning")


def save_table(table: dict, path: str) -> None:
    with open(path, "w") as f:
        json.dump({"version": 1, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
                   "buckets": {str(k): v for k, v in table.items()}}, f, indent=1)


def load_table(path: str) -> dict:
    if not os.path.exists(path):
        return {}
    d = json.load(open(path))
    return {int(k): v for k, v in d.get("buckets", {}).items()}


def tune(ctx, workloads, path=None, trace_depth=2, log=print, base=None) -> dict:
    """workloads: list of (scene_data, cameras) or (scene_data, cameras, trace_depth, spp).
    The buckets tuned replace those of the table at `base` (default `path`); returns the
    table and saves it at `path` when given."""
    src = base or path
    table = load_table(src) if src else {}
    for w in workloads:
        sc, cams = w[0], w[1]
        td = w[2] if len(w) > 2 else trace_depth
        spp = w[3] if len(w) > 3 else 1
        b = bucket_of(sc.n_tris)
        if log:
            log(f"bucket {b}: {sc.name} ({sc.n_tris} tris), {len(cams)} views, trace depth {td}, {spp} spp")
        table[b] = tune_scene(ctx, sc, cams, td, log=log, spp=spp)
    if path:
        save_table(table, path)
    apply_table(ctx, table)
    return table
