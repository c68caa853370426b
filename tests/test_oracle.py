"""CPU tests: the oracle pinned against the reference's golden vectors and, where the
reference tree is present, against the compiled reference itself."""
import os

import numpy as np
import pytest

import oracle
from eos_b200 import scenes
from tests.parity import RGB_TOL, classify, path_mismatch, primary_rays

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def test_morton_golden_vectors():
    """EncodeMorton3 (src/morton.h:45-48) outputs recorded from the compiled reference."""
    g = load("morton3")
    xyz = g["xyz"].astype(np.uint64)

    def spread(x):
        x = x & 0x3FF
        out = np.zeros_like(x)
        for b in range(10):
            out |= ((x >> b) & 1) << (3 * b)
        return out

    codes = (spread(xyz[:, 2]) << 2) + (spread(xyz[:, 1]) << 1) + spread(xyz[:, 0])
    assert np.array_equal(codes.astype(np.uint32), g["codes"])


def test_oracle_morton_order_is_stable_sort():
    sc = scenes.small_random_scene(3)
    codes, order = oracle.morton(sc.verts, sc.tris)
    keys = codes[order].astype(np.uint64) << 32 | order.astype(np.uint64)
    assert np.all(np.diff(keys.astype(np.int64)) > 0)
    # duplicate centroids: identical triangles keep id order
    v = np.zeros((3, 3), np.float32)
    v[1, 0] = 1
    v[2, 1] = 1
    tris = np.array([[0, 1, 2]] * 5, np.uint32)
    c, o = oracle.morton(v, tris)
    assert list(o) == [0, 1, 2, 3, 4] and len(set(c.tolist())) == 1


@pytest.mark.parametrize("name,scene_fn", [
    ("config1_128", lambda: scenes.config1_scene()),
    ("small11", lambda: scenes.small_random_scene(11, n_spheres=5, level=2, lights=3, refl=0.6)),
    ("small12", lambda: scenes.small_random_scene(12, n_spheres=5, level=2, lights=3, refl=0.6)),
    ("transp61", lambda: scenes.small_random_scene(61, n_spheres=6, level=2, lights=3, refl=0.5, transparent=3,
                                                   ambient_index=1.0002)),
    ("deep71", lambda: scenes.mirror_hall_scene(71)),  # trace depth 7, 8 lights
])
def test_oracle_matches_reference_golden(name, scene_fn):
    """Oracle paths and colours vs the reference's own renderer output (golden file)."""
    g = load(name)
    W, H, td = (int(v) for v in g["size"])
    cam = scenes.CameraData(*[g["cam"][3 * i:3 * i + 3] for i in range(4)], W, H)
    sc = scene_fn()
    r = oracle.Oracle(sc).render(cam, td, pixel_offset=0.0)
    nb = td + 1
    mm = path_mismatch(r["hits"], r["shadows"], g["hits"], g["shadows"], nb)
    c = classify(mm, r["flags"])
    assert c["unexplained"] == 0, c
    assert c["mismatch"] <= 0.002 * c["paths"], c
    d = np.abs(r["rgb"] - g["rgb"]).max(1)
    assert d[~mm].max() <= RGB_TOL
    # the restatement reproduces the reference's float colours exactly on matching paths
    assert (d[~mm] == 0).mean() > 0.999
    assert np.array_equal(r["counts"][0], g["counts"][0])


def test_oracle_matches_reference_config2_sample():
    """The oracle against the reference's renderer on 30,000 sampled paths of the
    1,056,768-triangle 1080p view (golden file recorded with the reference's own tree)."""
    path = os.path.join(os.path.dirname(__file__), "golden", "config2_sample.npz")
    if not os.path.exists(path):
        pytest.skip("config2_sample.npz not generated")
    g = np.load(path)
    sc = scenes.config2_scene()
    cam = scenes.config2_camera()
    r = oracle.Oracle(sc).render(cam, 2, pixel_offset=0.5, pixels=g["pixels"])
    mm = path_mismatch(r["hits"], r["shadows"], g["hits"], g["shadows"], 3)
    c = classify(mm, r["flags"])
    print("oracle vs reference, config 2 sample:", c)
    assert c["unexplained"] == 0, c
    assert np.abs(r["rgb"] - g["rgb"]).max(1)[~mm].max() <= RGB_TOL
    assert np.array_equal(r["counts"][0], g["counts"][0])


def test_oracle_matches_reference_config5_sample():
    """The oracle against the reference's renderer on 3,000 sampled paths of the
    4,524,288-triangle 4K stress view (depth 4, 8 lights, thin foliage triangles; golden file
    recorded with the reference's own tree)."""
    path = os.path.join(os.path.dirname(__file__), "golden", "config5_sample.npz")
    if not os.path.exists(path):
        pytest.skip("config5_sample.npz not generated")
    g = np.load(path)
    sc = scenes.config5_scene()
    cam = scenes.config5_camera()
    r = oracle.Oracle(sc).render(cam, 3, pixel_offset=0.5, pixels=g["pixels"])
    mm = path_mismatch(r["hits"], r["shadows"], g["hits"], g["shadows"], 4)
    c = classify(mm, r["flags"])
    print("oracle vs reference, config 5 sample:", c)
    assert c["unexplained"] == 0, c
    assert np.abs(r["rgb"] - g["rgb"]).max(1)[~mm].max() <= RGB_TOL
    assert np.array_equal(r["counts"][0], g["counts"][0])


@pytest.mark.parametrize("name", ["config3_job69", "config3_job0"])
def test_oracle_matches_reference_config3_jobs(name):
    """The oracle against the reference's renderer on 20,000 sampled paths of two jobs of
    the batching workload (its largest mixed scene, 361,330 triangles, and a 1080p view of
    the config-1 scene)."""
    path = os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{name}.npz not generated")
    g = np.load(path)
    j = scenes.config3_jobs()[int(g["job"])]
    r = oracle.Oracle(j.scene).render(j.camera, j.trace_depth, pixel_offset=j.pixel_offset, pixels=g["pixels"])
    mm = path_mismatch(r["hits"], r["shadows"], g["hits"], g["shadows"], j.trace_depth + 1)
    c = classify(mm, r["flags"])
    print(f"oracle vs reference, {name}:", c)
    assert c["unexplained"] == 0, c
    assert c["axis_parallel_not_tie"] + c["near_origin_not_tie"] <= 10, c
    assert np.abs(r["rgb"] - g["rgb"]).max(1)[~mm].max() <= RGB_TOL
    assert np.array_equal(r["counts"][0], g["counts"][0])


def test_oracle_matches_reference_config3_mixed_scenes():
    """The oracle against the reference's renderer on the other 15 mixed scenes of the
    batching workload (25k-315k triangles; 2,000 sampled paths of each, recorded on the
    trees the reference's builder made)."""
    g = load("config3_mixed")
    spec = scenes.config3_jobs()
    for k in np.unique(g["job"]):
        j = spec[int(k)]
        sel = g["job"] == k
        r = oracle.Oracle(j.scene).render(j.camera, j.trace_depth, pixel_offset=j.pixel_offset,
                                          pixels=g["pixels"][sel])
        mm = path_mismatch(r["hits"], r["shadows"], g["hits"][sel], g["shadows"][sel], j.trace_depth + 1)
        c = classify(mm, r["flags"])
        assert c["unexplained"] == 0, (int(k), c)
        assert c["axis_parallel_not_tie"] + c["near_origin_not_tie"] <= 5, (int(k), c)
        assert np.abs(r["rgb"] - g["rgb"][sel]).max(1)[~mm].max() <= RGB_TOL, int(k)


def test_oracle_matches_reference_config4_views():
    """The oracle against the reference's renderer on the differentiation workload's forward
    render: 4,000 sampled paths of each of its 8 views at 256^2 (config 4's scene with the
    shininess rounded down to the reference's int)."""
    g = load("config4_views")
    sc = scenes.integer_shininess(scenes.config4_scene())
    cams = scenes.config4_cameras(8, 256)
    o = oracle.Oracle(sc)
    shadow_rays = 0
    for v, cam in enumerate(cams):
        sel = g["view"] == v
        r = o.render(cam, 1, pixel_offset=0.5, pixels=g["pixels"][sel])
        mm = path_mismatch(r["hits"], r["shadows"], g["hits"][sel], g["shadows"][sel], 2)
        c = classify(mm, r["flags"])
        assert c["unexplained"] == 0, (v, c)
        assert c["axis_parallel_not_tie"] + c["near_origin_not_tie"] <= 5, (v, c)
        assert np.abs(r["rgb"] - g["rgb"][sel]).max(1)[~mm].max() <= RGB_TOL, v
        shadow_rays += int(r["counts"][1])
    assert shadow_rays == int(g["counts"][1])


def test_reference_tree_restore_equals_build():
    """The reference's tree exported after its own build and restored (boxes recomputed by
    BVH::computeBoxWithSurfaces) gives the same node buffer boxes and the same renders."""
    if not oracle.ref_available():
        pytest.skip("reference CPU build unavailable")
    sc = scenes.small_random_scene(71, n_spheres=8, level=3, lights=2, refl=0.5, transparent=1)
    built = oracle.RefRenderer(sc)
    perm, nodes = built.export_tree()
    restored = oracle.RefRenderer(sc, tree=(perm, nodes))
    assert restored.n_nodes == built.n_nodes and restored.max_leaf == built.max_leaf
    assert np.array_equal(built.boxes().view(np.uint32), restored.boxes().view(np.uint32))
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 64, 48)
    a, b = built.render(cam, 3), restored.render(cam, 3)
    assert np.array_equal(a["hits"], b["hits"]) and np.array_equal(a["shadows"], b["shadows"])
    assert np.array_equal(a["rgb"].view(np.uint32), b["rgb"].view(np.uint32))
    with pytest.raises(ValueError):  # a tree of another scene is refused
        oracle.RefRenderer(scenes.small_random_scene(72, n_spheres=2), tree=(perm, nodes))


@pytest.mark.parametrize("seed,ambient", [(62, 1.0), (63, 1.33), (64, 1.0002)])
def test_transparent_materials_match_reference(seed, ambient):
    """Transparent materials (src/RayTracer.cpp:353-407: Fresnel K, the mirror ray about the
    incident-side normal traced for both halves of the mix) against the compiled reference:
    paths and FP32 colours exact."""
    if not oracle.ref_available():
        pytest.skip("reference CPU build unavailable")
    sc = scenes.small_random_scene(seed, n_spheres=6, level=2, lights=3, refl=0.5, transparent=3,
                                   ambient_index=ambient)
    cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 80, 60)
    r = oracle.RefRenderer(sc).render(cam, 4, pixel_offset=0.0)
    o = oracle.Oracle(sc).render(cam, 4, pixel_offset=0.0)
    mm = path_mismatch(o["hits"], o["shadows"], r["hits"], r["shadows"], 5)
    assert classify(mm, o["flags"])["unexplained"] == 0
    assert np.abs(o["rgb"] - r["rgb"]).max(1)[~mm].max() <= RGB_TOL
    transparent_tris = np.nonzero(sc.materials[sc.tri_obj, 8] > 0)[0]
    assert np.isin(o["hits"][:, :4], transparent_tris).sum() > 100  # the case is exercised


def test_oracle_bvh_equals_brute_force():
    sc = scenes.small_random_scene(5, n_spheres=6, level=2)
    orc = oracle.Oracle(sc)
    cam = scenes.look_at((1, 2.5, 8), (0, 0, 0), 60, 48, 40)
    rays = primary_rays(cam, 0.5)
    rng = np.random.default_rng(1)
    rnd = np.concatenate([rng.uniform(-3, 3, (2000, 3)), rng.normal(size=(2000, 3))], 1).astype(np.float32)
    rnd[:, 3:] /= np.linalg.norm(rnd[:, 3:], axis=1, keepdims=True)
    # axis-parallel rays: exact zero direction components
    ax = np.zeros((300, 6), np.float32)
    ax[:, :3] = rng.uniform(-3, 3, (300, 3))
    ax[np.arange(300), 3 + rng.integers(0, 3, 300)] = rng.choice([-1.0, 1.0], 300)
    for R in (rays, rnd, ax):
        a, ta, _ = orc.closest(R)
        b, tb = orc.closest_brute(R)
        assert np.array_equal(a, b)
        assert np.array_equal(ta[a >= 0], tb[b >= 0])


def test_oracle_any_hit_semantics():
    sc = scenes.small_random_scene(6)
    orc = oracle.Oracle(sc)
    rng = np.random.default_rng(2)
    r = np.concatenate([rng.uniform(-3, 3, (3000, 3)), rng.normal(size=(3000, 3))], 1).astype(np.float32)
    r[:, 3:] /= np.linalg.norm(r[:, 3:], axis=1, keepdims=True)
    occ = orc.any(r)
    ids, _ = orc.closest_brute(r)
    assert np.array_equal(occ.astype(bool), ids >= 0)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU build unavailable")
def test_oracle_matches_compiled_reference_config1_full():
    """Full 512x512 config-1 frame: oracle vs the compiled reference renderer."""
    sc = scenes.config1_scene()
    cam = scenes.config1_camera()
    ref = oracle.RefRenderer(sc).render(cam, 1, pixel_offset=0.0)
    r = oracle.Oracle(sc).render(cam, 1, pixel_offset=0.0)
    mm = path_mismatch(r["hits"], r["shadows"], ref["hits"], ref["shadows"], 2)
    c = classify(mm, r["flags"])
    assert c["unexplained"] == 0, c
    d = np.abs(r["rgb"] - ref["rgb"]).max(1)
    assert d[~mm].max() <= RGB_TOL


@pytest.mark.parametrize("spp", [1, 2])
def test_frozen_f64_adjoint_matches_central_differences(spp):
    """FP64 analytic adjoint vs central differences (step 1e-3) of the FP64 frozen render;
    with 2 jittered samples per pixel, the pixel is their mean."""
    sc = scenes.small_random_scene(21, n_spheres=4, level=2, lights=2, refl=0.4)
    cams = [scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 24, 20),
            scenes.look_at((-6.0, 4.0, 6.0), (0, -0.5, 0), 55.0, 24, 20)]
    orc = oracle.Oracle(sc)
    td = 2
    seed = 5
    hits, shadows = [], []
    for c in cams:
        r = orc.render(c, td, pixel_offset=0.5, spp=spp, jitter_seed=seed)
        hits.append(r["hits"])
        shadows.append(r["shadows"])
    hits = np.concatenate(hits)
    shadows = np.concatenate(shadows)
    mp = sc.materials.astype(np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    lp = sc.lights.astype(np.float64).copy()
    rng = np.random.default_rng(3)
    target = rng.uniform(0, 0.5, (len(cams) * 24 * 20, 3))

    def loss(m, l):
        rgb = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, m, l, spp=spp, jitter_seed=seed)
        return float(((rgb - target) ** 2).sum()), rgb

    L0, rgb = loss(mp, lp)
    if spp > 1:  # the FP64 mean of the samples is the FP32 forward's colour, up to rounding
        r32 = np.concatenate([orc.render(c, td, pixel_offset=0.5, spp=spp, jitter_seed=seed)["rgb"] for c in cams])
        assert np.abs(rgb - r32).max() < 1e-3
    g = 2.0 * (rgb - target)
    _, gm, gl = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, mp, lp, g=g, spp=spp, jitter_seed=seed)
    h = 1e-3
    checks = [("m", 0, 0), ("m", 1, 4), ("m", 2, 6), ("m", 4, 2), ("l", 0, 0), ("l", 1, 4), ("l", 0, 3), ("l", 1, 5)]
    for kind, i, j in checks:
        m2, l2 = mp.copy(), lp.copy()
        arr = m2 if kind == "m" else l2
        orig = arr[i, 3 + j if kind == "l" and j < 3 else (j - 3 if kind == "l" else j)]
        col = (3 + j) if (kind == "l" and j < 3) else ((j - 3) if kind == "l" else (j if j < 6 else 6))
        arr[i, col] = orig + h
        Lp, _ = loss(m2 if kind == "m" else mp, l2 if kind == "l" else lp)
        arr[i, col] = orig - h
        Lm, _ = loss(m2 if kind == "m" else mp, l2 if kind == "l" else lp)
        fd = (Lp - Lm) / (2 * h)
        an = gm[i, j] if kind == "m" else gl[i, j]
        assert abs(fd - an) <= 1e-3 * max(1.0, abs(fd)), (kind, i, j, fd, an)


def test_instanced_oracle_agrees_with_the_flattened_scene():
    """The two-level restatement (rays moved into object space) against the same triangles
    transformed into world space in float64: the same nearest triangles but where two
    candidates lie within rounding of each other, colours within 1e-4 elsewhere."""
    d = scenes.instanced_test_scene(13, n_instances=10, lights=2)
    cam = scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 64, 48)
    a = oracle.OracleInstanced(d).render(cam, 2, pixel_offset=0.5)
    b = oracle.Oracle(d.flatten()).render(cam, 2, pixel_offset=0.5)
    same = (a["hits"][:, :3] == b["hits"][:, :3]).all(1)
    assert same.mean() > 0.995
    assert np.abs(a["rgb"] - b["rgb"]).max(1)[same].max() < 1e-4
    assert (a["hits"][:, 0] >= 0).mean() > 0.2


def test_reference_builder_bounds_placed_triangles():
    """The reference's own builder over object-space triangles with per-object
    transformations (eosref_scene_create_transformed, as its main program places a mesh):
    every leaf box holds its placed triangles under translations and axis scales (the
    placements the GPU comparison uses), and not under a rotation -- its
    Box::transformBoundingBox moves only the local box's two corners (src/Box.cu:84-135)."""
    if not oracle.ref_available():
        pytest.skip("reference CPU build unavailable")
    from oracle import ref_gpu
    d, _ = ref_gpu.transformed_case()
    verts, normals, tris, tri_mat, tri_xf, xf = ref_gpu.object_space_arrays(d)
    sc = scenes.SceneData(verts, normals, tris, tri_mat, d.materials, d.lights)

    def leaves_outside(xforms):
        """Placed triangles outside their leaf's box, and the root box."""
        r = oracle.RefRenderer(sc, transforms=(tri_xf, xforms))
        perm, nodes = r.export_tree()
        boxes = r.boxes().astype(np.float64)
        M = np.asarray(xforms, np.float64).reshape(-1, 3, 4)
        out = 0
        for i in np.nonzero(nodes[:, 0] == 1)[0]:  # BVH_LEAF (src/BVH.h:34-37)
            ids = perm[nodes[i, 4]:nodes[i, 4] + nodes[i, 1]]
            for t in ids:
                p = verts[tris[t]].astype(np.float64) @ M[tri_xf[t], :, :3].T + M[tri_xf[t], :, 3]
                out += int(((p < boxes[i, :3] - 1e-5) | (p > boxes[i, 3:] + 1e-5)).any())
        return out, boxes[0]

    out, root = leaves_outside(xf)
    assert out == 0
    world = d.flatten().verts.astype(np.float64)
    assert np.allclose(root[:3], world.min(0), rtol=0, atol=1e-5)
    assert np.allclose(root[3:], world.max(0), rtol=0, atol=1e-5)
    c, s_ = np.cos(np.pi / 4), np.sin(np.pi / 4)
    xr = xf.copy().reshape(-1, 3, 4)
    xr[4, :, :3] = xr[4, :, :3] @ np.array([[c, 0, s_], [0, 1, 0], [-s_, 0, c]], np.float32)
    out_r, _ = leaves_outside(xr.reshape(-1, 12))
    assert out_r > 0


def test_instanced_frozen_f64_adjoint_matches_central_differences():
    """The FP64 adjoint of a two-level scene (hits replayed in each instance's object space,
    normals through the inverse transpose) against central differences of its own FP64
    frozen render."""
    d = scenes.instanced_test_scene(7, n_instances=8, lights=2)
    d.materials[:, 7] = 0.3
    orc = oracle.OracleInstanced(d)
    cams = [scenes.look_at((1.0, 3.0, 9.0), (0, -0.5, 0), 55.0, 24, 20)]
    td = 2
    r = orc.render(cams[0], td, pixel_offset=0.5)
    hits, shadows = r["hits"], r["shadows"]
    assert (hits[:, 0] >= 0).mean() > 0.3
    mp = np.asarray(d.materials, np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    lp = np.asarray(d.lights, np.float64).copy()
    target = np.random.default_rng(5).uniform(0, 0.5, (24 * 20, 3))

    def loss(m, l):
        rgb = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, m, l)
        return float(((rgb - target) ** 2).sum()), rgb

    _, rgb = loss(mp, lp)
    assert np.abs(rgb - r["rgb"]).max() < 1e-3  # FP64 replay of the FP32 frame
    _, gm, gl = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, mp, lp, g=2.0 * (rgb - target))
    h = 1e-3
    for kind, i, col, gcol in [("m", 1, 0, 0), ("m", 2, 4, 4), ("m", 3, 6, 6), ("l", 0, 3, 0), ("l", 1, 0, 3)]:
        arr = (mp if kind == "m" else lp).copy()
        arr[i, col] += h
        Lp, _ = loss(arr, lp) if kind == "m" else loss(mp, arr)
        arr[i, col] -= 2 * h
        Lm, _ = loss(arr, lp) if kind == "m" else loss(mp, arr)
        fd = (Lp - Lm) / (2 * h)
        an = gm[i, gcol] if kind == "m" else gl[i, gcol]
        assert abs(fd - an) <= 1e-3 * max(1.0, abs(fd)), (kind, i, col, fd, an)


def test_ploc_restatement_small_cases():
    """The PLOC restatement on hand-checked inputs: two pairs of unit boxes far apart merge
    pairwise, then into the root; any input gives a permutation with contiguous subtrees."""
    from oracle import ploc
    lo = np.array([[0, 0, 0], [1, 0, 0], [10, 0, 0], [11, 0, 0]], np.float32)
    child, count, pos = ploc.build(lo, lo + 1)
    assert child.tolist() == [[3, 4], [5, 6], [0, 1]] and count.tolist() == [2, 2, 4]
    assert pos.tolist() == [0, 1, 2, 3]
    child, count, pos = ploc.build(lo[:2], lo[:2] + 1)
    assert child.tolist() == [[1, 2]] and pos.tolist() == [0, 1]
    rng = np.random.default_rng(3)
    c = rng.uniform(-5, 5, (700, 3)).astype(np.float32)
    child, count, pos = ploc.build(c, c + rng.uniform(0, 1, (700, 3)).astype(np.float32))
    n = 700
    assert sorted(pos.tolist()) == list(range(n)) and count[n - 2] == n
    leaves = {}
    for k in range(n - 1):  # children are made before their parents
        s = []
        for c in child[k]:
            assert c >= n - 1 or c < k
            s += [c - (n - 1)] if c >= n - 1 else leaves[c]
        leaves[k] = s
        p = np.sort(pos[s])
        assert p[-1] - p[0] + 1 == len(s) == count[k]  # each subtree a contiguous range


# ----------------------------------------------------------------------------- ray trees
def tree_scene():
    return scenes.small_random_scene(91, n_spheres=7, level=2, lights=3, refl=0.5, transparent=1, both=3,
                                     ambient_index=1.0002)


def test_oracle_tree_matches_reference_golden():
    """Materials both reflective and transparent: the reference traces both secondary rays
    (src/RayTracer.cpp:339-407).  The oracle's ray trees (heap order) and FP32 colours vs
    the reference's own renderer (golden file both91.npz): bit-exact."""
    g = load("both91")
    W, H, td = (int(v) for v in g["size"])
    cam = scenes.CameraData(*[g["cam"][3 * i:3 * i + 3] for i in range(4)], W, H)
    r = oracle.Oracle(tree_scene()).render_tree(cam, td, pixel_offset=0.0)
    assert r["hits"].shape[1] == oracle.tree_nodes(td) == 15
    mm = (r["hits"] != g["hits"]).any(1) | (r["shadows"] != g["shadows"]).any(1)
    c = classify(mm, r["flags"])
    assert c["unexplained"] == 0 and c["mismatch"] == 0, c
    assert np.array_equal(r["rgb"].view(np.uint32), g["rgb"].view(np.uint32))
    assert np.array_equal(r["counts"], g["counts"])
    # the case is exercised: paths whose hits on both children of one node were traced
    both = ((r["hits"][:, 1:15:2] != -2) & (r["hits"][:, 2:15:2] != -2)).any(1)
    assert both.sum() > 50


def test_oracle_tree_render_equals_chain_render_on_chain_scenes():
    """Without such materials the tree form holds the chain: same colours bit for bit, same
    ray counts, and every chain bounce's record at its node."""
    sc = scenes.small_random_scene(11, n_spheres=5, level=2, lights=3, refl=0.6, transparent=2)
    cam = scenes.look_at((0.5, 3.0, 9.0), (0, -0.5, 0), 55.0, 64, 48)
    orc = oracle.Oracle(sc)
    a = orc.render(cam, 3, pixel_offset=0.5)
    b = orc.render_tree(cam, 3, pixel_offset=0.5)
    assert np.array_equal(a["rgb"].view(np.uint32), b["rgb"].view(np.uint32))
    assert np.array_equal(a["counts"], b["counts"])
    mats = sc.materials[sc.tri_obj]  # per-triangle material rows
    for p in range(a["hits"].shape[0]):
        node = 0
        for k in range(4):
            assert b["hits"][p, node] == a["hits"][p, k] and b["shadows"][p, node] == a["shadows"][p, k]
            h = a["hits"][p, k]
            if h < 0 or k == 3:
                break
            node = 2 * node + (1 if mats[h, 7] > 0 else 2)


def test_frozen_f64_tree_adjoint_matches_central_differences():
    """The FP64 adjoint over ray trees (mirror edge weight = reflectivity, transparent edge
    weight 1) vs central differences of the FP64 frozen tree render, and its colours vs the
    FP32 tree render."""
    sc = tree_scene()
    cams = [scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 24, 20)]
    orc = oracle.Oracle(sc)
    td = 3
    r = orc.render_tree(cams[0], td, pixel_offset=0.5)
    hits, shadows = r["hits"], r["shadows"]
    mp = sc.materials.astype(np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    lp = sc.lights.astype(np.float64).copy()
    target = np.random.default_rng(4).uniform(0, 0.5, (24 * 20, 3))

    def loss(m, l):
        rgb = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, m, l, tree=True)
        return float(((rgb - target) ** 2).sum()), rgb

    L0, rgb = loss(mp, lp)
    assert np.abs(rgb - r["rgb"]).max() < 1e-3
    g = 2.0 * (rgb - target)
    _, gm, gl = orc.frozen_f64(cams, 24, 20, 0.5, td, hits, shadows, mp, lp, g=g, tree=True)
    h = 1e-3
    for kind, i, col in [("m", 1, 0), ("m", 2, 4), ("m", 3, 6), ("m", 7, 1), ("l", 0, 3), ("l", 1, 0), ("l", 2, 5)]:
        m2, l2 = mp.copy(), lp.copy()
        arr = m2 if kind == "m" else l2
        orig = arr[i, col]
        arr[i, col] = orig + h
        Lp, _ = loss(m2, l2)
        arr[i, col] = orig - h
        Lm, _ = loss(m2, l2)
        fd = (Lp - Lm) / (2 * h)
        an = gm[i, col] if kind == "m" else gl[i, col - 3 if col >= 3 else col + 3]
        assert abs(fd - an) <= 1e-3 * max(1.0, abs(fd)), (kind, i, col, fd, an)


def test_oracle_aa_grid_matches_reference_golden():
    """The reference's anti-aliasing grid (RayTracer::renderWithAA, src/RayTracer.cpp:176-265,
    3 x 3 samples): per-sample paths and FP32 colours bit-exact, and the reference's own
    RGBA8 frame equals the oracle's colours quantised (golden aa3_small12.npz)."""
    g = load("aa3_small12")
    W, H, td, n = (int(v) for v in g["size"])
    cam = scenes.CameraData(*[g["cam"][3 * i:3 * i + 3] for i in range(4)], W, H)
    sc = scenes.small_random_scene(12, n_spheres=5, level=2, lights=3, refl=0.6)
    o = oracle.Oracle(sc).render(cam, td, spp=n * n, aa_grid=True)
    assert np.array_equal(o["hits"][:, :td + 1], g["hits"]) and np.array_equal(o["shadows"][:, :td + 1], g["shadows"])
    assert np.array_equal(o["rgb"].view(np.uint32), g["rgb"].view(np.uint32))
    assert np.array_equal(o["counts"], g["counts"])
    c = o["rgb"].reshape(H, W, 3).astype(np.float64)
    q = np.floor(np.where(c == 1.0, 255, np.minimum(c * 256.0, 255.0))).astype(np.uint8)
    assert np.array_equal(q, g["rgba8"][..., :3])
    with pytest.raises(ValueError):
        oracle.grid_side(5)
