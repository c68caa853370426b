"""Generates the golden fixtures in this directory from the reference's own CPU code.

Runs the reference renderer compiled from its sources (oracle/_ref/libeosref.so, built by
oracle/Makefile from the reference tree) and its EncodeMorton3 on seeded inputs and
stores the outputs as small .npz files.  The GPU box has no reference tree, so the
tests read these files there.

    python tests/golden/make_golden.py            (all fixtures)
    python tests/golden/make_golden.py config2    (the 1.06M-triangle sample only)
    python tests/golden/make_golden.py trees      (the ray-tree scene only)
    python tests/golden/make_golden.py aa         (the anti-aliasing grid case only)
    python tests/golden/make_golden.py deep       (the deepest paths: trace depth 7, 8 lights)
    python tests/golden/make_golden.py config5    (the 4.5M-triangle 4K sample only)
    python tests/golden/make_golden.py config3    (two jobs of the batching workload only)
    python tests/golden/make_golden.py config4    (the differentiation workload's 8 views only)
    python tests/golden/make_golden.py config3mixed  (the other 15 mixed scenes of the batching workload)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from eos_b200 import scenes  # noqa: E402


def render_case(name, scene, cam, trace_depth):
    ref = oracle.RefRenderer(scene, build_threads=1)
    r = ref.render(cam, trace_depth, pixel_offset=0.0, nthreads=os.cpu_count())
    nb = trace_depth + 1
    rgba8, _ = ref.render_rgba8(cam, trace_depth, nthreads=os.cpu_count())
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), rgb=r["rgb"], hits=r["hits"][:, :nb],
                        shadows=r["shadows"][:, :nb].astype(np.uint8 if scene.n_lights <= 8 else np.uint32),
                        counts=r["counts"], rgba8=rgba8, cam=cam.as_array(),
                        size=np.array([cam.width, cam.height, trace_depth]),
                        ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
    print(name, r["counts"], "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def morton_case():
    rng = np.random.default_rng(7)
    xyz = rng.integers(0, 1024, size=(4096, 3), dtype=np.uint32)
    edge = np.array([[0, 0, 0], [1023, 1023, 1023], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1023, 0, 0],
                     [0, 1023, 0], [0, 0, 1023], [512, 256, 128], [2047, 4095, 1024]], np.uint32)
    xyz = np.concatenate([edge, xyz])
    codes = oracle.ref_morton3(xyz)
    np.savez_compressed(os.path.join(HERE, "morton3.npz"), xyz=xyz, codes=codes)
    print("morton3", codes[:10])


def tree_scene():
    """Spheres whose materials are both reflective and transparent (each hit on them spawns
    two secondary rays) beside a transparent one and mirrors, in air."""
    return scenes.small_random_scene(91, n_spheres=7, level=2, lights=3, refl=0.5, transparent=1, both=3,
                                     ambient_index=1.0002)


def tree_case():
    """Ray-tree records (heap order) and FP32 colours of the reference on tree_scene()."""
    sc = tree_scene()
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 96, 72)
    td = 3
    ref = oracle.RefRenderer(sc, build_threads=1)
    r = ref.render_tree(cam, td, pixel_offset=0.0, nthreads=os.cpu_count())
    np.savez_compressed(os.path.join(HERE, "both91.npz"), rgb=r["rgb"], hits=r["hits"],
                        shadows=r["shadows"].astype(np.uint8), counts=r["counts"], cam=cam.as_array(),
                        size=np.array([cam.width, cam.height, td]), ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
    print("both91", r["counts"], "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def aa_case():
    """The reference's anti-aliasing grid (RayTracer::setAASamples(3), renderWithAA): FP32
    colours, per-sample paths and the reference's own RGBA8 frame."""
    sc = scenes.small_random_scene(12, n_spheres=5, level=2, lights=3, refl=0.6)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 48, 36)
    td, n = 2, 3
    ref = oracle.RefRenderer(sc, build_threads=1)
    r = ref.render_aa(cam, td, n, nthreads=os.cpu_count())
    rgba8, _ = ref.render_rgba8(cam, td, nthreads=os.cpu_count(), aa=n)
    np.savez_compressed(os.path.join(HERE, "aa3_small12.npz"), rgb=r["rgb"], hits=r["hits"][:, :td + 1],
                        shadows=r["shadows"][:, :td + 1].astype(np.uint8), counts=r["counts"], rgba8=rgba8,
                        cam=cam.as_array(), size=np.array([cam.width, cam.height, td, n]))
    print("aa3_small12", r["counts"])


def deep_case():
    render_case("deep71", scenes.mirror_hall_scene(71), scenes.look_at((-0.3, 0.5, 5.0), (1.2, -0.6, -3.0), 60.0, 80, 60), 7)


def config2_case(n_sample=30_000):
    """30,000 seeded pixels of the 1080p view of the 1,056,768-triangle scene (depth 3, 4
    lights, pixel centres) through the reference's renderer, with the tree its own builder
    made (saved once by oracle/make_ref_tree.py and restored here)."""
    from oracle import make_ref_tree
    sc = scenes.config2_scene()
    tree = make_ref_tree.load(sc)
    if tree is None:
        raise SystemExit("run `python -m oracle.make_ref_tree` first (builds the reference's tree once)")
    ref = oracle.RefRenderer(sc, tree=tree)
    cam = scenes.config2_camera()
    rng = np.random.default_rng(2002)
    pix = np.sort(rng.choice(cam.width * cam.height, n_sample, replace=False)).astype(np.int32)
    r = ref.render(cam, 2, pixel_offset=0.5, pixels=pix, nthreads=os.cpu_count())
    np.savez_compressed(os.path.join(HERE, "config2_sample.npz"), pixels=pix, rgb=r["rgb"], hits=r["hits"][:, :3],
                        shadows=r["shadows"][:, :3].astype(np.uint8), counts=r["counts"], cam=cam.as_array(),
                        size=np.array([cam.width, cam.height, 2]), ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
    print("config2_sample", r["counts"], "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def config5_case(n_sample=3_000):
    """3,000 seeded pixel centres of the 4K view of the 4,524,288-triangle stress scene
    (depth 4, 8 lights; one sample at each pixel centre -- the reference has no jittered
    samples) through the reference's renderer, with the tree its own builder made (saved
    once by `python -m oracle.make_ref_tree --scene config5`)."""
    from oracle import make_ref_tree
    sc = scenes.config5_scene()
    tree = make_ref_tree.load(sc, "config5")
    if tree is None:
        raise SystemExit("run `python -m oracle.make_ref_tree --scene config5` first")
    ref = oracle.RefRenderer(sc, tree=tree)
    cam = scenes.config5_camera()
    rng = np.random.default_rng(5005)
    pix = np.sort(rng.choice(cam.width * cam.height, n_sample, replace=False)).astype(np.int32)
    r = ref.render(cam, 3, pixel_offset=0.5, pixels=pix, nthreads=os.cpu_count())
    np.savez_compressed(os.path.join(HERE, "config5_sample.npz"), pixels=pix, rgb=r["rgb"], hits=r["hits"][:, :4],
                        shadows=r["shadows"][:, :4].astype(np.uint8), counts=r["counts"], cam=cam.as_array(),
                        size=np.array([cam.width, cam.height, 3]), ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
    print("config5_sample", r["counts"], "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def config3_case(n_sample=20_000):
    """Two jobs of the batching workload (scenes.config3_jobs): its largest mixed scene
    (job 69, 361,330 triangles, 512^2, 20,000 seeded pixel centres) and its first view of
    the config-1 scene (job 0, 1920x1080 from 120 units away, 20,000 seeded pixel centres of
    the central 600 x 600 pixels, where the scene is), depth 3, through the reference's
    renderer on trees its own builder made (single-threaded; config 1's from oracle/_ref)."""
    from oracle import make_ref_tree
    jobs = scenes.config3_jobs()
    rng = np.random.default_rng(3003)
    for k, name in ((69, "config3_job69"), (0, "config3_job0")):
        j = jobs[k]
        tree = make_ref_tree.load(j.scene, "config1") if k == 0 else None
        ref = oracle.RefRenderer(j.scene, build_threads=1, tree=tree)
        cam = j.camera
        if k == 0:
            xs, ys = np.meshgrid(np.arange(cam.width // 2 - 300, cam.width // 2 + 300),
                                 np.arange(cam.height // 2 - 300, cam.height // 2 + 300))
            pool = (ys * cam.width + xs).reshape(-1)
        else:
            pool = np.arange(cam.width * cam.height)
        pix = np.sort(rng.choice(pool, n_sample, replace=False)).astype(np.int32)
        r = ref.render(cam, j.trace_depth, pixel_offset=j.pixel_offset, pixels=pix, nthreads=os.cpu_count())
        nb = j.trace_depth + 1
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), job=np.array(k), pixels=pix, rgb=r["rgb"],
                            hits=r["hits"][:, :nb], shadows=r["shadows"][:, :nb].astype(np.uint8),
                            counts=r["counts"], cam=cam.as_array(),
                            size=np.array([cam.width, cam.height, j.trace_depth]),
                            ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
        print(name, r["counts"], "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def _config3_mixed_job(args):
    """One mixed scene of the batching workload through the reference's renderer (run in a
    worker process: the reference's builder is single-threaded)."""
    k, n_sample = args
    j = scenes.config3_jobs()[k]
    ref = oracle.RefRenderer(j.scene, build_threads=1)
    cam = j.camera
    pix = np.sort(np.random.default_rng(3100 + k).choice(cam.width * cam.height, n_sample,
                                                          replace=False)).astype(np.int32)
    r = ref.render(cam, j.trace_depth, pixel_offset=j.pixel_offset, pixels=pix, nthreads=1)
    nb = j.trace_depth + 1
    return (k, pix, r["rgb"], r["hits"][:, :nb], r["shadows"][:, :nb].astype(np.uint8), np.asarray(r["counts"]),
            ref.n_nodes, ref.max_leaf)


def config3_mixed_case(n_sample=2_000):
    """The other 15 mixed scenes of the batching workload (jobs 64-79 but 69, 25k-315k
    triangles, 512^2, depth 3, 2 lights): 2,000 seeded pixel centres of each through the
    reference's renderer on the tree its own builder makes, one worker process per scene."""
    import multiprocessing as mp
    jobs = scenes.config3_jobs()
    ks = [k for k, j in enumerate(jobs) if j.scene.name.startswith("mixed") and k != 69]
    with mp.get_context("spawn").Pool(min(len(ks), os.cpu_count() or 1)) as pool:
        res = pool.map(_config3_mixed_job, [(k, n_sample) for k in ks])
    res.sort(key=lambda t: t[0])
    out = dict(job=np.concatenate([np.full(len(t[1]), t[0], np.int32) for t in res]),
               pixels=np.concatenate([t[1] for t in res]), rgb=np.concatenate([t[2] for t in res]),
               hits=np.concatenate([t[3] for t in res]), shadows=np.concatenate([t[4] for t in res]),
               counts=np.stack([t[5] for t in res]), ref_nodes=np.array([[t[6], t[7]] for t in res]))
    np.savez_compressed(os.path.join(HERE, "config3_mixed.npz"), **out)
    for t in res:
        print("config3 job", t[0], t[5], "nodes", t[6], "max leaf", t[7])


def config4_case(n_per_view=4_000):
    """The differentiation workload's forward render: all 8 views at 256^2 of config 4's
    scene (50 level-3 icospheres on a ground quad, 3 lights, depth 2 = trace depth 1),
    4,000 seeded pixel centres per view, through the reference's renderer on the tree its
    own builder makes (single-threaded).  The reference's shininess is an int, so the scene
    is config 4 with each shininess rounded down (scenes.integer_shininess)."""
    sc = scenes.integer_shininess(scenes.config4_scene())
    cams = scenes.config4_cameras(8, 256)
    ref = oracle.RefRenderer(sc, build_threads=1)
    rng = np.random.default_rng(4004)
    out = {k: [] for k in ("view", "pixels", "rgb", "hits", "shadows")}
    counts = np.zeros(3, np.int64)
    for v, cam in enumerate(cams):
        pix = np.sort(rng.choice(cam.width * cam.height, n_per_view, replace=False)).astype(np.int32)
        r = ref.render(cam, 1, pixel_offset=0.5, pixels=pix, nthreads=os.cpu_count())
        out["view"].append(np.full(n_per_view, v, np.int32))
        out["pixels"].append(pix)
        out["rgb"].append(r["rgb"])
        out["hits"].append(r["hits"][:, :2])
        out["shadows"].append(r["shadows"][:, :2].astype(np.uint8))
        counts += np.asarray(r["counts"][:3], np.int64)
    np.savez_compressed(os.path.join(HERE, "config4_views.npz"), **{k: np.concatenate(v) for k, v in out.items()},
                        counts=counts, size=np.array([256, 256, 1]), ref_nodes=np.array([ref.n_nodes, ref.max_leaf]))
    print("config4_views", counts, "nodes", ref.n_nodes, "max leaf", ref.max_leaf)


def main():
    oracle.build(ref=True)
    if sys.argv[1:] == ["config4"]:
        config4_case()
        return
    if sys.argv[1:] == ["config3mixed"]:
        config3_mixed_case()
        return
    if sys.argv[1:] == ["config2"]:
        config2_case()
        return
    if sys.argv[1:] == ["trees"]:
        tree_case()
        return
    if sys.argv[1:] == ["aa"]:
        aa_case()
        return
    if sys.argv[1:] == ["deep"]:
        deep_case()
        return
    if sys.argv[1:] == ["config5"]:
        config5_case()
        return
    if sys.argv[1:] == ["config3"]:
        config3_case()
        return
    morton_case()
    render_case("config1_128", scenes.config1_scene(), scenes.config1_camera(128, 128), 1)
    for seed in (11, 12):
        sc = scenes.small_random_scene(seed, n_spheres=5, level=2, lights=3, refl=0.6)
        cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 96, 72)
        render_case(f"small{seed}", sc, cam, 3)
    # transparent spheres (Fresnel-mixed secondary rays) in air
    sc = scenes.small_random_scene(61, n_spheres=6, level=2, lights=3, refl=0.5, transparent=3, ambient_index=1.0002)
    render_case("transp61", sc, scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 96, 72), 4)
    tree_case()
    aa_case()
    deep_case()
    config2_case()
    config5_case()
    config3_case()
    config3_mixed_case()
    config4_case()


if __name__ == "__main__":
    main()
