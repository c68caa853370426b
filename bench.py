"""Benchmark of the render path: Mrays/s at 1080p on the ~1.06M-triangle scene.

Default (one GPU): the 1,056,768-triangle scene (128x128-cell height field + 200 level-4
icospheres, 4 lights, depth 3), V views at 1920x1080, 1 spp at pixel centres.  One step
renders the V views:

  value   batched persistent wavefront (one eos_render_batch call = one CUDA-graph replay
          of all V views), outputs resident in HBM, CUDA events on the library stream
  plain   the same V views as V one-launch-per-frame eos_render calls (reported beside)
  e2e     the public API with host memory: one eos_render_batch call per step whose jobs
          write pinned host RGBA8 images (job table in, images out), queued with
          EOS_FLAG_ASYNC so that each step's copy to the host overlaps the next step's
          rendering, wall clock from the first call to eos_ctx_synchronize after the last;
          beside it the same calls synchronous, and the reference-facing per-frame call,
          eos_render once per view into a pinned host buffer (the DeviceRenderer::
          renderCudaSceneToHostBufferMegaKernel contract)

Rays = primary + shadow + secondary (mirror) rays actually traced, from the library's
counters.  The scene (~135 MB of node / triangle / shading records) is larger than L2.

--impl reference: the reference's own CPU renderer (compiled from its sources into
oracle/_ref/libeosref.so) on all host cores for the same metric and view: RayTracer::rayTrace
per pixel over a strided sample of the view's pixels per step, with the tree the reference's builder made for this
scene (built once, saved as oracle/_ref/config2_tree.npz and restored; the build takes ~10
minutes on one core).  The cpu_baseline of the GPU line is the same measurement, with the
oracle's C port beside it.

Multi-GPU (torchrun, N ranks): views are independent, every rank renders its own V views
(weak scaling, no data-path collective); timing = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s @1080p 1M tris, batched vs plain GPU; fwd+adjoint ms/view"
TUNING = os.path.join(ROOT, "eos_b200", "tuning_b200.json")


def run_autotune(only=None, out=None):
    """Tunes one representative workload per scene-size bucket and writes the table (to
    `out`, default the committed table); `only`: names of the workloads to tune, the other
    buckets are kept as they are."""
    import numpy as np
    from eos_b200 import api, autotune, scenes
    ctx = api.Context(0)
    rng = scenes.rng_for(4242)
    work = {"config1": lambda: (scenes.config1_scene(), [scenes.config1_camera()]),
            "mixed60k": lambda: (scenes.mixed_scene(rng, 60_000, "mixed60k"),
                                 [scenes.look_at((0, 25, 60), (0, 0, 0), 60.0, 512, 512)]),
            "mixed300k": lambda: (scenes.mixed_scene(rng, 300_000, "mixed300k"),
                                  [scenes.look_at((0, 25, 60), (0, 0, 0), 60.0, 512, 512)]),
            "config2": lambda: (scenes.config2_scene(), views_for(0, 4)),
            # the 4K stress view: depth 4 (trace depth 3), 2 jittered samples per pixel
            "config5": lambda: (scenes.config5_scene(), [scenes.config5_camera()], 3, 2)}
    names = list(work) if not only else [n for n in work if n in only]
    if only and len(names) != len(set(only)):
        raise SystemExit(f"--autotune-only takes {', '.join(work)}")
    if only:  # the generators draw from one stream: make the skipped ones too, in order
        items = []
        for n in work:
            w = work[n]()
            if n in names:
                items.append(w)
    else:
        items = [work[n]() for n in names]
    table = autotune.tune(ctx, items, path=out or TUNING, trace_depth=2, base=TUNING)
    print(json.dumps({str(k): {"setting": v["setting"], "mrays": round(v["mrays"], 1),
                               "default_mrays": round(v["default_mrays"], 1)} for k, v in table.items()}))
    del np


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--views", type=int, default=4)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU megakernel as a comparison point")
    ap.add_argument("--no-config3", action="store_true", help="skip the 80-job batching workload")
    ap.add_argument("--no-config5", action="store_true", help="skip the 4.5M-triangle 4K stress workload")
    ap.add_argument("--profile", action="store_true",
                    help="profiling case for ncu: one 1080p view, batched and plain steps only")
    ap.add_argument("--autotune", action="store_true",
                    help=f"tune block / queue chunk / stack depth / leaf size per scene-size bucket and "
                         f"write {os.path.relpath(TUNING, ROOT)}")
    ap.add_argument("--autotune-only", nargs="+", default=None,
                    help="with --autotune: the workloads to tune (config1 mixed60k mixed300k config2 config5)")
    ap.add_argument("--tuning-out", default=None, help="with --autotune: write the table here instead")
    ap.add_argument("--no-tuning", action="store_true", help="ignore the committed tuning table")
    a = ap.parse_args()
    if a.profile:
        a.views, a.no_adjoint, a.no_cpu_baseline, a.no_config3, a.no_config5 = 1, True, True, True, True
        a.no_reference_gpu = True
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def views_for(rank: int, n: int):
    """Camera orbit around the config-2 target; rank r gets its own views (weak scaling)."""
    import math
    from eos_b200 import scenes
    cams = []
    for v in range(n):
        a = 2 * math.pi * (rank * n + v) / max(8, n) * 0.25
        if rank == 0 and v == 0:
            cams.append(scenes.config2_camera())
            continue
        cams.append(scenes.look_at((160 * math.sin(a), 60, 160 * math.cos(a)), (0, 0, 0), 60.0, 1920, 1080))
    return cams


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nme, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nme)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(st, width):
    """Algorithmic bytes of the shadow (any-hit) and nearest-hit stages from the traversal
    counters: 32 B per ray in; 4 B out per shadow ray, 16 B per nearest hit; 28 B per child
    box visited (an AABB and a reference; a node visit reads `width` of them); 40 B per
    triangle test (three vertices and an id); 84 B per shaded hit (normals 36 B, material
    32 B, colour read-modify-write 16 B).  Layout-independent floor: what a node or
    triangle record holds beyond this (padding, counts) is not counted."""
    node = 28 * width
    shadow = (32 + 4) * st["shadow_rays"] + node * st["nodes_shadow"] + 40 * st["tests_shadow"]
    closest = ((32 + 16) * (st["primary_rays"] + st["secondary_rays"]) + node * st["nodes_closest"]
               + 40 * st["tests_closest"] + 84 * st["shaded_hits"])
    return shadow, closest


def profile_traffic():
    """Per-ray counters of the top kernels from the committed ncu summary (profiles/traffic.json):
    warp instructions, L1 / L2 / DRAM bytes per ray, and the per-cycle peaks of the part."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return {}


def roofline(tr, st, stage_ms, shadow_bytes, closest_bytes, launches, sm_hz):
    """Roofline of the wavefront's two traversal stages against the ceiling that binds them.

    Both are gathers through a tree whose node and triangle records are mostly served by L1
    and L2, not streams from HBM; the ncu captures show instruction issue as the limit
    (issue slots ~70 % busy, 18-25 of 32 lanes active per instruction).  So the headline
    fraction is issue: warp instructions per ray (ncu capture of the same kernel) x this
    step's rays of the stage / the stage's CUDA-event time, against the part's issue peak
    (sm__inst_issued.sum.peak_sustained = 592 warp instructions per cycle) at the SM clock
    sampled under load.  Beside it the same rays' L1, L2 and DRAM bytes against their peaks
    (ncu per-cycle peaks; HBM: the measured copy bandwidth), and the algorithmic bytes."""
    hbm_peak, hbm_kind = measured_peak()
    peaks = tr.get("peaks_per_cycle", {})
    out = {}
    for key, kern, ms, alg, rays in (
            ("shadow", "k_wf_any", stage_ms[1], shadow_bytes, st["shadow_rays"]),
            ("closest", "k_wf_closest", stage_ms[0], closest_bytes, st["primary_rays"] + st["secondary_rays"])):
        c = tr.get(key)
        sec = ms * 1e-3
        e = {"kernel": kern, "stage_ms": round(ms, 4), "launches": launches, "rays": rays,
             "ms_per_launch": round(ms / launches, 4),
             "algorithmic_bytes_per_launch": round(alg / launches),
             "algorithmic_note": "node / triangle record bytes requested (28 B per child box, 40 B per test, "
                                 "32 B ray in, result out): an L1-level request count, mostly served by L1 / L2"}
        if c and peaks:
            inst = c["warp_inst_per_ray"] * rays
            issue_peak = peaks["issue_warp_inst"] * sm_hz
            l1_peak = peaks["l1_bytes"] * sm_hz
            l2_peak = peaks["l2_bytes"] * peaks["l2_clock_hz"]
            e.update({
                "bound": "issue", "achieved": round(inst / sec / 1e9, 1),
                "peak": round(issue_peak / 1e9, 1), "unit": "Gwarp-inst/s",
                "frac": round(inst / sec / issue_peak, 4),
                "peak_kind": "ncu sm__inst_issued.sum.peak_sustained (592 warp instructions per cycle) x the "
                             "median SM clock sampled during this run",
                "traffic": round(c["dram_bytes_per_ray"] * rays / launches),
                "traffic_source": "ncu capture of the same kernel: DRAM bytes per ray x rays per launch "
                                  "(cold caches: an upper bound)",
                "ceilings": {
                    "issue": round(inst / sec / issue_peak, 4),
                    "l1_bytes": round(c["l1_bytes_per_ray"] * rays / sec / l1_peak, 4),
                    "l2_bytes": round(c["l2_bytes_per_ray"] * rays / sec / l2_peak, 4),
                    "hbm_bytes": round(c["dram_bytes_per_ray"] * rays / sec / (hbm_peak * 1e9), 4)},
                "hbm_peak_gbs": hbm_peak, "hbm_peak_kind": hbm_kind,
                "per_ray": {k: c[k] for k in ("warp_inst_per_ray", "l1_bytes_per_ray", "l2_bytes_per_ray",
                                              "dram_bytes_per_ray")},
                "ncu": {k: c[k] for k in ("issue_active_pct", "l1tex_throughput_pct", "threads_per_warp_instruction",
                                          "warps_active_pct")}})
        out[key] = e
    top = max(out, key=lambda k: out[k]["stage_ms"])
    roof = dict(out[top])
    roof["stages"] = {k: {x: v for x, v in out[k].items() if x not in ("algorithmic_note", "peak_kind",
                                                                        "traffic_source")} for k in out}
    roof["stage_ms"] = [round(x, 3) for x in stage_ms]
    return roof


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_renderer(sc):
    """The reference's own CPU renderer over scene sc with the tree its builder made for it
    (saved once by oracle/make_ref_tree.py), or None when that tree file is absent."""
    import oracle
    from oracle import make_ref_tree
    if not oracle.ref_available():
        return None
    tree = make_ref_tree.load(sc)
    if tree is None:
        return None
    return oracle.RefRenderer(sc, tree=tree)


def ref_sample(ref, cam, trace_depth, target_s, nthreads):
    """Pixels spread evenly over the whole view (every k-th pixel), as many as the reference's
    RayTracer::rayTrace renders in about target_s seconds on nthreads threads, and their ray
    count (primary + shadow + secondary, replayed once outside any timing).  The reference
    is slow on this scene (its depth-limited tree has leaves of up to 438 triangles), so the
    sample is a small strided subset of the frame."""
    import numpy as np
    n = cam.width * cam.height

    def strided(count):
        step = max(1, n // max(1, count))
        return np.arange(step // 2, n, step, dtype=np.int32)[:count]

    probe = strided(512)
    r = ref.render(cam, trace_depth, pixel_offset=0.5, pixels=probe, nthreads=nthreads, paths=False)
    count = int(min(n, max(256, len(probe) * target_s / max(r["seconds"], 1e-3))))
    pix = strided(count)
    counts = ref.render(cam, trace_depth, pixel_offset=0.5, pixels=pix, nthreads=nthreads)["counts"]
    return pix, int(counts.sum())


def ref_timed(ref, cam, trace_depth, pix, nthreads):
    r = ref.render(cam, trace_depth, pixel_offset=0.5, pixels=pix, nthreads=nthreads, paths=False)
    return r["seconds"]


def cpu_baseline(sc, cam, trace_depth, budget_s=15.0):
    """The reference's own CPU renderer on all host threads on a bounded band of rows
    (kind "reference"), with the oracle's C port on a sample of the same view beside it."""
    nthreads = os.cpu_count()
    port = port_baseline(sc, cam, trace_depth, budget_s=min(budget_s, 6.0))
    ref = ref_renderer(sc)
    if ref is None:
        port["note"] = "reference tree file absent (oracle/make_ref_tree.py): the port is reported"
        return port
    pix, rays = ref_sample(ref, cam, trace_depth, budget_s / 4.0, nthreads)
    secs = [ref_timed(ref, cam, trace_depth, pix, nthreads) for _ in range(3)]
    sec = statistics.median(secs)
    return {"value": rays / sec / 1e6, "unit": "Mrays/s", "cores": nthreads, "kind": "reference",
            "cpu": cpu_model(),
            "sample": f"{len(pix)} pixels spread evenly over the 1080p view ({rays} rays) through the reference's "
                      f"RayTracer::rayTrace (oracle/_ref/libeosref.so, the tree of its own builder), "
                      f"{nthreads} threads, median of 3",
            "rays": rays, "seconds": sec,
            "port": {"value": round(port["value"], 3), "unit": "Mrays/s", "cores": port["cores"],
                     "sample": port["sample"]}}


def port_baseline(sc, cam, trace_depth, budget_s=15.0):
    """The oracle's C port of the render path on all host threads, on a bounded sample of rows."""
    import numpy as np
    import oracle
    orc = oracle.Oracle(sc)
    nthreads = os.cpu_count()
    W, H = cam.width, cam.height
    rows = 8
    total_rays, total_t, rows_done = 0, 0.0, 0
    y0 = H // 2 - 64
    while total_t < budget_s and rows_done < H:
        pix = np.arange((y0 + rows_done) * W, (y0 + rows_done + rows) * W, dtype=np.int32) % (W * H)
        t = time.perf_counter()
        r = orc.render(cam, trace_depth, pixel_offset=0.5, pixels=pix, nthreads=nthreads)
        total_t += time.perf_counter() - t
        total_rays += int(r["counts"].sum())
        rows_done += rows
        rows = min(rows * 2, 128)
    return {"value": total_rays / total_t / 1e6, "unit": "Mrays/s", "cores": nthreads, "kind": "port",
            "sample": f"{rows_done} rows x {W} px of the 1080p view (oracle C port, {nthreads} threads)",
            "rays": total_rays, "seconds": total_t}


def reference_gpu_point(scene: str, reps: int = 5, timeout_s: int = 300):
    """The reference's own GPU megakernel (primary rays and local Phong only) on this GPU, as
    a comparison point: `python -m oracle.ref_gpu` in a process of its own (the reference
    exits on any CUDA error)."""
    try:
        r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", "--scene", scene, "--reps", str(reps)],
                           cwd=ROOT, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"timed out after {timeout_s} s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"unavailable": f"exit {r.returncode}: " + (r.stderr.strip().splitlines() or [""])[-1][:200]}
    return json.loads(lines[-1])


def run_reference(args, rank, world):
    """The reference's own CPU renderer on the host cores for the same metric and view: one
    step = a strided sample of the 1080p view's pixels (about 3 s of work) through
    RayTracer::rayTrace, all host threads; the tree is the one the reference's builder made for this scene,
    restored from oracle/_ref/config2_tree.npz (the build itself takes ~10 min on one core)."""
    if rank != 0:
        return
    from eos_b200 import scenes
    sc = scenes.config2_scene()
    cam = scenes.config2_camera()
    nthreads = os.cpu_count()
    ref = ref_renderer(sc)
    workload = ("1920x1080 view of the 1,056,768-tri scene (height field 128^2 + 200 level-4 icospheres), "
                "depth 3, 4 lights, 1 spp at pixel centres")
    if ref is not None:
        pix, rays = ref_sample(ref, cam, 2, 3.0, nthreads)
        secs = []
        for i in range(args.warmup + args.steps):
            sec = ref_timed(ref, cam, 2, pix, nthreads)
            if i >= args.warmup:
                secs.append(sec)
        v = rays * len(secs) / sum(secs) / 1e6
        cpu = {"value": v, "unit": "Mrays/s", "cores": nthreads, "kind": "reference", "cpu": cpu_model(),
               "sample": f"per step {len(pix)} pixels spread evenly over the view ({rays} rays) through the "
                         f"reference's RayTracer::rayTrace (oracle/_ref/libeosref.so, the tree of its own "
                         f"builder)"}
    else:
        res, info = [], None
        for i in range(args.warmup + args.steps):
            info = port_baseline(sc, cam, 2, budget_s=4.0)
            if i >= args.warmup:
                res.append(info["value"])
        v = statistics.median(res)
        cpu = {"value": v, "unit": "Mrays/s", "cores": info["cores"], "kind": "port", "cpu": cpu_model(),
               "sample": info["sample"] + " per step; the reference's tree file oracle/_ref/config2_tree.npz "
                                          "is absent"}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": workload, "mode": "CPU"},
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        import datetime
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    if args.autotune:
        if rank == 0:
            run_autotune(args.autotune_only, args.tuning_out)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    run_ours(args, rank, world, local)


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    from eos_b200 import api, scenes

    dev = local
    torch.cuda.set_device(dev)
    ctx = api.Context(dev)
    tuned = False
    if not args.no_tuning and os.path.exists(TUNING):
        from eos_b200 import autotune
        autotune.apply_table(ctx, autotune.load_table(TUNING))
        tuned = True
    sc = scenes.config2_scene()
    dsc = api.DeviceScene(ctx, sc, inputs_on_device=True)
    info = dsc.info()
    # the first build of a process also allocates the builder's scratch; a repeat build of
    # the same scene is the steady-state cost
    rebuild_ms = api.DeviceScene(ctx, sc, inputs_on_device=True).info()["build_ms"]
    cams = views_for(rank, args.views)
    td = 2
    jobs = [api.BatchJob(dsc, c, td, 0.5) for c in cams]
    outs = api.make_batch_outputs(jobs, ("rgba8",))
    plain_out = [{"rgba8": o["rgba8"]} for o in outs]
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)

    def step_batched():
        return api.render_batch(ctx, jobs, outs)

    def step_plain():
        st = []
        for c, o in zip(cams, plain_out):
            st.append(api.render(ctx, dsc, c, td, pixel_offset=0.5, outputs=(), out=dict(o))["stats"])
        return st

    def rays_of(s):
        return s["primary_rays"] + s["shadow_rays"] + s["secondary_rays"]

    def sync_all():
        torch.cuda.synchronize(dev)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, steps):
        sync_all()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        rays, launches = 0, 0
        for _ in range(steps):
            s = fn()
            ss = s if isinstance(s, list) else [s]
            rays += sum(rays_of(x) for x in ss)
            launches += sum(x["kernel_launches"] for x in ss)
        ev1.record(stream)
        sync_all()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ms], device=f"cuda:{dev}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t)
            r = torch.tensor([float(rays)], device=f"cuda:{dev}", dtype=torch.float64)
            dist.all_reduce(r)
            rays = float(r)
        return ms, rays, launches

    b0 = None
    if args.profile:
        # bounce 0 of view 0 alone, before anything else: the launches that an ncu capture with
        # -s 0 -c 1 of k_wf_closest / k_wf_any sees, so its DRAM bytes divide by known ray counts
        b0 = api.render_batch(ctx, [api.BatchJob(dsc, cams[0], 0, 0.5)], outs[:1])

    # clocks are sampled every 200 ms from the warm-up to the end of the GPU measurements
    clk = ClockSampler(dev).__enter__()
    for _ in range(args.warmup):
        step_batched()
        step_plain()
    ms_b, rays_b, launches_b = timed(step_batched, args.steps)
    ms_p, rays_p, launches_p = timed(step_plain, args.steps)
    mrays_b = rays_b / (ms_b * 1e-3) / 1e6
    mrays_p = rays_p / (ms_p * 1e-3) / 1e6
    if args.profile:
        clk.__exit__(None, None, None)
        if rank == 0:
            print(json.dumps({"profile_case": True, "batched_mrays": round(mrays_b, 1),
                              "plain_mrays": round(mrays_p, 1),
                              "bounce0": {k: b0[k] for k in ("primary_rays", "shadow_rays", "nodes_closest",
                                                             "tests_closest", "nodes_shadow", "tests_shadow",
                                                             "shaded_hits")}}), flush=True)
        return

    # e2e through the public API with pinned host outputs, host<->device copies inside the
    # timed region: (a) one eos_render_batch call per step for all views (the headline);
    # (b) the reference-facing per-frame call, eos_render once per view
    host_imgs = [torch.empty((c.height, c.width, 4), dtype=torch.uint8).pin_memory() for c in cams]
    host_outs = [{"rgba8": h} for h in host_imgs]
    def step_e2e_batch():
        return [api.render_batch(ctx, jobs, host_outs)]

    def step_e2e_view(mode):
        st = []
        for c, h in zip(cams, host_imgs):
            st.append(api.render(ctx, dsc, c, td, pixel_offset=0.5, mode=mode, outputs=(),
                                 out={"rgba8": h.numpy()}, device=False)["stats"])
        return st

    def wall_timed(fn):
        for _ in range(max(1, args.warmup)):
            fn()
        sync_all()
        t0 = time.perf_counter()
        rays_e = 0
        for _ in range(args.steps):
            rays_e += sum(rays_of(s) for s in fn())
        sync_all()
        e2e_s = time.perf_counter() - t0
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s, float(rays_e)], device=f"cuda:{dev}", dtype=torch.float64)
            tm = t.clone()
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
            dist.all_reduce(t)
            e2e_s, rays_e = float(tm[0]), float(t[1])
        return rays_e / e2e_s / 1e6

    e2e_sync = wall_timed(step_e2e_batch)

    def e2e_pipelined():
        """The same calls with EOS_FLAG_ASYNC: each call returns once queued, its copy of the
        images to the pinned host buffers overlaps the next call's rendering, and the timed
        region ends when eos_ctx_synchronize has every copy done (rays per call from the
        stats that the synchronize returns)."""
        for _ in range(max(1, args.warmup)):
            api.render_batch(ctx, jobs, host_outs, async_outputs=True)
        ctx.synchronize()
        sync_all()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            api.render_batch(ctx, jobs, host_outs, async_outputs=True)
        stats = ctx.synchronize()
        sync_all()
        e2e_s = time.perf_counter() - t0
        rays_e = float(sum(rays_of(x) for x in stats))
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s, rays_e], device=f"cuda:{dev}", dtype=torch.float64)
            tm = t.clone()
            dist.all_reduce(tm, op=dist.ReduceOp.MAX)
            dist.all_reduce(t)
            e2e_s, rays_e = float(tm[0]), float(t[1])
        return rays_e / e2e_s / 1e6

    e2e = e2e_pipelined()
    e2e_modes = {m: wall_timed(lambda: step_e2e_view(m)) for m in ("plain", "wavefront")}
    e2e_mode = max(e2e_modes, key=e2e_modes.get)
    e2e_view = e2e_modes[e2e_mode]

    # roofline of the dominant kernel: per-stage device time of the wavefront (eager, one step)
    st = api.render_batch(ctx, jobs, outs, stage_timing=True)
    shadow_bytes, closest_bytes = algorithmic_bytes(st, info["width"])
    stage = st["stage_ms"]
    # the stage-timed run launches its stages one by one in a single lane: one launch per
    # bounce per chunk; the library's chunk rule: at most 2^24 paths (8x4-pixel tiles) and at
    # most 16 GB of queues at (2 x 32 + 2 x (36 + 32 x lights) + 16 x (depth + 1)) B per path
    paths = sum(((c.width + 7) // 8) * ((c.height + 3) // 4) * 32 for c in cams)
    per_path = 2 * 32 + 2 * (36 + 32 * max(1, sc.n_lights)) + 16 * (td + 1)
    chunk = max(1 << 16, min(1 << 24, (16 << 30) // per_path))
    launches_stage = (td + 1) * int(np.ceil(paths / float(chunk)))
    sm_hz = (clk.summary()["sm_mhz"] or 1965.0) * 1e6
    roof = roofline(profile_traffic(), st, stage, shadow_bytes, closest_bytes, launches_stage, sm_hz)

    # adjoint: forward (with path records) + backward per view, config-4 style parameters
    adj = None
    if not args.no_adjoint:
        adj = adjoint_timing(ctx, stream)

    batch3 = None
    if not args.no_config3:
        batch3 = config3_timing(ctx, stream, max(2, args.steps // 2), max(1, args.warmup))
    stress5 = None
    if not args.no_config5:
        stress5 = config5_timing(ctx, stream, 2, 1)
    clk.__exit__(None, None, None)
    clocks = clk.summary()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc, cams[0], td)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = {"config2_1080p": reference_gpu_point("config2"), "config1_512": reference_gpu_point("config1")}
        ref_gpu["note"] = ("the reference's __rayTrace_MegaKernel compiled for sm_100a (oracle/_ref/libeosref_gpu.so): "
                           "one primary ray per pixel and local Phong over all lights, no shadow or mirror rays, on "
                           "its own tree; a comparison point, not this line's workload (which traces shadow and "
                           "mirror rays as the reference's CPU renderer does)")

    npx_step = sum(c.width * c.height for c in cams)
    line = {
        "metric": METRIC, "value": round(mrays_b, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_b / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"{len(cams)} views/GPU at 1920x1080 of the 1,056,768-tri scene "
                               "(height field 128^2 + 200 level-4 icospheres), depth 3, 4 lights, 1 spp",
                   "mode": "batched persistent wavefront, CUDA graph", "l2": "inputs larger than L2 (scene records "
                   f"{info['device_bytes'] / 1e6:.0f} MB)", "leaf_size": info["leaf_size"],
                   "tuning": "eos_b200/tuning_b200.json" if tuned else "defaults"},
        "plain": {"value": round(mrays_p, 2), "unit": "Mrays/s", "ms_per_step": round(ms_p / args.steps, 3)},
        "batched_over_plain": round(mrays_b / mrays_p, 3),
        "rays_per_step": {"total": rays_b / args.steps / world},
        # the headline split by ray type: this rank's per-step counts at the whole-job step time
        "mrays_by_type": {k: round(st[k + "_rays"] * world / (ms_b / args.steps * 1e-3) / 1e6, 2)
                          for k in ("primary", "shadow", "secondary")},
        "e2e": {"value": round(e2e, 2), "unit": "Mrays/s",
                "call": "eos_render_batch with EOS_FLAG_ASYNC per step, all views, pinned host RGBA8 outputs; "
                        "each step's copy to the host overlaps the next step's rendering; wall clock from the "
                        "first call to eos_ctx_synchronize after the last",
                "h2d_bytes_per_step": len(cams) * 184 + 36, "d2h_bytes_per_step": 4 * npx_step,
                "synchronous_call": {"value": round(e2e_sync, 2),
                                     "call": "the same eos_render_batch without EOS_FLAG_ASYNC (returns with the "
                                             "images on the host)"},
                "per_view_call": {"value": round(e2e_view, 2), "call": f"eos_render per view, {e2e_mode} mode",
                                  "modes": {m: round(v, 2) for m, v in e2e_modes.items()}}},
        "gpu_launches": launches_b,
        "roofline": roof,
        "clocks": clocks,
        "build_ms": round(info["build_ms"], 3),
        "rebuild_ms": round(rebuild_ms, 3),
        "builder": {1: "lbvh", 2: "ploc"}.get(info["builder"], "?"),
        "bvh": {"layout": {1: "sah", 2: "fixed"}.get(info["layout"], "?"), "leaf_size": info["leaf_size"],
                "sah_cost": round(info["sah_cost"], 2), "width": info["width"], "node_records": info["n_nodes"],
                "scene_device_mb": round(info["device_bytes"] / 1e6, 1)},
        "traversal_per_ray": {
            "nearest_nodes": round(st["nodes_closest"] / max(1, st["primary_rays"] + st["secondary_rays"]), 2),
            "nearest_tests": round(st["tests_closest"] / max(1, st["primary_rays"] + st["secondary_rays"]), 2),
            "shadow_nodes": round(st["nodes_shadow"] / max(1, st["shadow_rays"]), 2),
            "shadow_tests": round(st["tests_shadow"] / max(1, st["shadow_rays"]), 2),
            "rays": {"primary": st["primary_rays"], "shadow": st["shadow_rays"], "secondary": st["secondary_rays"]}},
    }
    if adj:
        line["adjoint"] = adj
    if batch3:
        line["config3_batch"] = batch3
    if stress5:
        line["config5_stress"] = stress5
    if ref_gpu:
        line["reference_gpu_kernel"] = ref_gpu
    if cpu:
        line["cpu_baseline"] = {k: (float(f"{v:.4g}") if isinstance(v, float) else v) for k, v in cpu.items()
                                if k in ("value", "unit", "cores", "kind", "sample", "cpu", "port", "note")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.set_stream(None)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def config3_timing(ctx, stream, steps, warmup):
    """Batching workload: 64 views of the config-1 scene at mixed resolutions plus 16 mixed
    scenes (10k-500k tris) at 512^2, depth 3, as one eos_render_batch call (graph replay)
    against one eos_render call per view."""
    import torch
    from eos_b200 import api, scenes
    spec = scenes.config3_jobs()
    dev = {}
    jobs = []
    for j in spec:
        if id(j.scene) not in dev:
            dev[id(j.scene)] = api.DeviceScene(ctx, j.scene, inputs_on_device=True)
        jobs.append(api.BatchJob(dev[id(j.scene)], j.camera, j.trace_depth, j.pixel_offset))
    outs = api.make_batch_outputs(jobs, ("rgba8",))

    def batched():
        return [api.render_batch(ctx, jobs, outs)]

    def plain():
        return [api.render(ctx, j.scene, j.camera, j.trace_depth, j.pixel_offset, outputs=(), out=dict(o))["stats"]
                for j, o in zip(jobs, outs)]

    res = {}
    for name, fn in (("batched", batched), ("plain", plain)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rays = 0
        for _ in range(steps):
            rays += sum(s["primary_rays"] + s["shadow_rays"] + s["secondary_rays"] for s in fn())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = {"mrays": round(rays / (ms * 1e-3) / 1e6, 1), "ms_per_step": round(ms / steps, 3)}
    n_tris = sorted({j.scene.n_tris for j in spec})
    return {"jobs": len(jobs), "scenes": len(dev), "tris_range": [n_tris[0], n_tris[-1]],
            "pixels": sum(j.camera.width * j.camera.height for j in spec), **res,
            "batched_over_plain": round(res["batched"]["mrays"] / res["plain"]["mrays"], 3)}


def config5_timing(ctx, stream, steps, warmup):
    """Stress workload: 3840x2160, 2 spp with jitter, depth 4, 8 lights, 4,524,288 thin
    triangles; one frame per step, batched wavefront vs plain.  The same scene also as
    801 instances (the height field once, the 5,000-triangle cluster stored once and placed
    800 times; eos_scene_create_instanced)."""
    import torch
    from eos_b200 import api, scenes
    sc = scenes.config5_scene()
    dsc = api.DeviceScene(ctx, sc, inputs_on_device=True)
    cam = scenes.config5_camera()

    def measure(scene):
        job = [api.BatchJob(scene, cam, 3, 0.5, spp=2, jitter_seed=7)]
        outs = api.make_batch_outputs(job, ("rgba8",))

        def batched():
            return [api.render_batch(ctx, job, outs)]

        def plain():
            return [api.render(ctx, scene, cam, 3, pixel_offset=0.5, spp=2, jitter_seed=7, outputs=(),
                               out=dict(outs[0]))["stats"]]

        res = {}
        for name, fn in (("batched", batched), ("plain", plain)):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rays = 0
            for _ in range(steps):
                rays += sum(s["primary_rays"] + s["shadow_rays"] + s["secondary_rays"] for s in fn())
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            res[name] = {"mrays": round(rays / (ms * 1e-3) / 1e6, 1), "ms_per_frame": round(ms / steps, 2),
                         "rays_per_frame": rays // steps}
        res["batched_over_plain"] = round(res["batched"]["mrays"] / res["plain"]["mrays"], 3)
        return res

    res = measure(dsc)
    info = dsc.info()
    out = {"tris": sc.n_tris, "resolution": "3840x2160", "spp": 2, "depth": 4, "lights": 8, **res,
           "build_ms": round(info["build_ms"], 2), "builder": {1: "lbvh", 2: "ploc"}.get(info["builder"], "?"),
           "scene_device_mb": round(info["device_bytes"] / 1e6, 1)}
    out["forward_adjoint"] = config5_adjoint(ctx, stream, dsc, cam)
    del dsc
    idata = scenes.config5_instanced()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    meshes = [api.DeviceScene(ctx, m, inputs_on_device=True) for m in idata.meshes]
    inst = api.InstancedScene(ctx, meshes, idata.instances, idata.materials, idata.lights)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    r2 = measure(inst)
    out["instanced"] = {"instances": len(idata.instances), "stored_tris": sum(m.n_tris for m in idata.meshes),
                        "scene_device_mb": round((inst.info()["device_bytes"] +
                                                  sum(m.info()["device_bytes"] for m in meshes)) / 1e6, 1),
                        "build_ms_wall": round(build_s * 1e3, 1), **r2}
    return out


def config5_adjoint(ctx, stream, dsc, cam, reps=2):
    """One forward + adjoint pass at config-5 scale: the 4K frame at 2 jittered samples, depth
    4, 8 lights, path records kept (one eos_render_batch), then eos_render_backward of an
    image loss gradient; ms per frame of each."""
    import torch
    from eos_b200 import api
    npx = cam.width * cam.height
    job = [api.BatchJob(dsc, cam, 3, 0.5, spp=2, jitter_seed=7)]
    outs = [{"rgb": torch.empty((npx, 3), device="cuda"),
             "paths": torch.empty((npx * 2, 16), dtype=torch.int32, device="cuda")}]
    g = torch.full((npx, 3), 0.01, device="cuda")

    def fwd():
        api.render_batch(ctx, job, outs)

    def bwd():
        api.render_backward(ctx, dsc, [cam], 3, outs[0]["paths"], g, pixel_offset=0.5, spp=2, jitter_seed=7)

    res = {}
    for name, fn in (("fwd", fwd), ("bwd", bwd)):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps
    return {"fwd_ms": round(res["fwd"], 2), "fwd_adj_ms": round(res["fwd"] + res["bwd"], 2),
            "ratio": round((res["fwd"] + res["bwd"]) / res["fwd"], 3),
            "calls": "eos_render_batch with path records (2 spp) + eos_render_backward"}


def adjoint_timing(ctx, stream, reps=5):
    """Differentiation workload (config 4): 8 views at 256^2 of 50 level-3 icospheres on a
    ground quad, 3 lights, depth 2.  fwd = the views rendered with path records; fwd+adj adds
    eos_render_backward of an image loss gradient; ms per view, for one batched call of each
    (the headline) and for one call per view."""
    import torch
    from eos_b200 import api, scenes

    def measure(dsc, cams, td):
        outs = []
        for c in cams:
            npx = c.width * c.height
            outs.append({"rgb": torch.empty((npx, 3), device="cuda"),
                         "paths": torch.empty((npx, 16), dtype=torch.int32, device="cuda")})
        g = [torch.full((c.width * c.height, 3), 0.01, device="cuda") for c in cams]

        def fwd():
            for c, o in zip(cams, outs):
                api.render(ctx, dsc, c, td, pixel_offset=0.5, outputs=(), out=dict(o))

        def fwdbwd():
            fwd()
            for c, o, gg in zip(cams, outs, g):
                api.render_backward(ctx, dsc, [c], td, o["paths"], gg, pixel_offset=0.5)

        npx = cams[0].width * cams[0].height
        paths_all = torch.empty((len(cams) * npx, 16), dtype=torch.int32, device="cuda")
        g_all = torch.full((len(cams) * npx, 3), 0.01, device="cuda")
        jobs = [api.BatchJob(dsc, c, td, 0.5) for c in cams]
        bouts = [{"rgb": torch.empty((npx, 3), device="cuda"), "paths": paths_all[i * npx:(i + 1) * npx]}
                 for i in range(len(cams))]

        def fwd_b():
            api.render_batch(ctx, jobs, bouts)

        def fwdbwd_b():
            fwd_b()
            api.render_backward(ctx, dsc, cams, td, paths_all, g_all, pixel_offset=0.5)

        res = {}
        for name, fn in (("fwd", fwd), ("fwd_adj", fwdbwd), ("fwd_b", fwd_b), ("fwd_adj_b", fwdbwd_b)):
            fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            res[name] = e0.elapsed_time(e1) / reps / len(cams)
        return {"fwd_ms_per_view": round(res["fwd_b"], 4), "fwd_adj_ms_per_view": round(res["fwd_adj_b"], 4),
                "ratio": round(res["fwd_adj_b"] / res["fwd_b"], 3),
                "calls": "one eos_render_batch with path records + one eos_render_backward for all views",
                "per_view_calls": {"fwd_ms_per_view": round(res["fwd"], 4),
                                   "fwd_adj_ms_per_view": round(res["fwd_adj"], 4),
                                   "ratio": round(res["fwd_adj"] / res["fwd"], 3),
                                   "calls": "eos_render (plain) + eos_render_backward per view"},
                "views": f"{len(cams)} x {cams[0].width}x{cams[0].height}"}

    sc4 = scenes.config4_scene()
    d4 = api.DeviceScene(ctx, sc4, inputs_on_device=True)
    out = measure(d4, scenes.config4_cameras(8, 256), 1)
    out["workload"] = "config 4: 50 ico3 + quad, 3 lights, depth 2"
    return out


if __name__ == "__main__":
    main()
