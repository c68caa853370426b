"""Known answers worked out by hand: Morton codes of points placed on the quantisation
grid, Moller-Trumbore hits with exact t / u / v, the |det| < 1e-5 rejection of thin
triangles, rays behind the origin, exact ties (larger id wins), unbounded shadow rays, and
an icosphere hit from its outside.  The oracle must give them on the CPU; the GPU test
asks the library the same questions."""
import numpy as np
import pytest

import oracle
from eos_b200 import scenes

MAT = np.array([[0.5, 0.5, 0.5, 0.2, 0.2, 0.2, 16, 0.0]], np.float32)
LIGHT = np.array([[0, 0, 10, 1, 1, 1]], np.float32)


def _scene(tris_xyz):
    v = np.asarray(tris_xyz, np.float32).reshape(-1, 3)
    n = np.tile([[0, 0, 1]], (len(v), 1)).astype(np.float32)
    t = np.arange(len(v), dtype=np.uint32).reshape(-1, 3)
    return scenes.SceneData(v, n, t, np.zeros(len(t)), MAT, LIGHT)


def _ray(o, d):
    return np.array([list(o) + list(d)], np.float32)


# Three triangles collapsed to points (centroid ((p + p) + p) / 3 = p exactly) at the
# corners and inside the unit cube: q = min(1023, floor(1024 (c - lo) / (hi - lo))).
#   (0, 0, 0)          -> q = (0, 0, 0)          -> code 0
#   (1, 1, 1)          -> q = (1023, 1023, 1023) -> code 0x3FFFFFFF
#   (0.5, 0.25, 0.75)  -> q = (512, 256, 768)    -> x bit 9 -> 1 << 27, y bit 8 -> 1 << 25,
#                         z bits 9, 8 -> 1 << 29 | 1 << 26: code 0x2E000000
POINTS = [(0, 0, 0), (1, 1, 1), (0.5, 0.25, 0.75)]
CODES = [0x00000000, 0x3FFFFFFF, 0x2E000000]


def _point_scene():
    return _scene([p for p in POINTS for _ in range(3)])


def test_morton_codes_by_hand():
    sc = _point_scene()
    codes, order = oracle.morton(sc.verts, sc.tris)
    assert [int(c) for c in codes] == CODES
    assert list(order) == [0, 2, 1]


def test_morton_flat_axis_quantises_to_zero():
    sc = _scene([(0, 0, 2)] * 3 + [(1, 0.5, 2)] * 3)
    codes, _ = oracle.morton(sc.verts, sc.tris)
    # x: 0 and 1023, y: 0 and 1023 (only two values), z: flat -> 0
    assert [int(c) for c in codes] == [0, 0x1B6DB6DB]


TRI = [(-1, -1, 0), (1, -1, 0), (0, 1, 0)]


def test_triangle_hit_exact_t():
    """MT by hand: e1 = (2,0,0), e2 = (1,2,0), d = (0,0,-1): P = (2,-1,0), det = 4,
    T = (1,1,5), Q = (0,10,-2), t = 20/4 = 5, u = 1/4, v = 2/4."""
    orc = oracle.Oracle(_scene(TRI))
    ids, t, _ = orc.closest(_ray((0, 0, 5), (0, 0, -1)))
    assert ids[0] == 0 and t[0] == 5.0
    ids, t, _ = orc.closest(_ray((0, 0, -5), (0, 0, 1)))   # from behind: det = -4, t = 5
    assert ids[0] == 0 and t[0] == 5.0
    ids, _, _ = orc.closest(_ray((0, 0, 5), (0, 0, 1)))    # pointing away: t = -5 < 0
    assert ids[0] == -1
    ids, _, _ = orc.closest(_ray((0, 0, 5), (1, 0, 0)))    # parallel to the plane: det = 0
    assert ids[0] == -1
    ids, _, _ = orc.closest(_ray((2, 0, 5), (0, 0, -1)))   # outside the edge: u > 1
    assert ids[0] == -1


@pytest.mark.parametrize("leg,hit", [(1e-3, False), (1e-2, True)])
def test_thin_triangle_det_threshold(leg, hit):
    """A right triangle of leg a seen along -z has det = a^2: 1e-6 is rejected by
    |det| < 1e-5 (src/Triangle.cpp:65), 1e-4 is not."""
    a = leg
    orc = oracle.Oracle(_scene([(0, 0, 0), (a, 0, 0), (0, a, 0)]))
    ids, _, _ = orc.closest(_ray((a / 4, a / 4, 1), (0, 0, -1)))
    assert (ids[0] == 0) == hit


def test_exact_tie_goes_to_the_larger_id():
    orc = oracle.Oracle(_scene(TRI + TRI + TRI))
    ids, t, _ = orc.closest(_ray((0, 0, 5), (0, 0, -1)))
    assert ids[0] == 2 and t[0] == 5.0


def test_shadow_rays_are_unbounded():
    """Any triangle at t >= 0 blocks, also beyond the light: a light at z = 1 above a
    triangle at z = 3 is still blocked for a point at z = 0 looking up."""
    orc = oracle.Oracle(_scene([(-1, -1, 3), (1, -1, 3), (0, 1, 3)]))
    assert orc.any(_ray((0, 0, 0), (0, 0, 1)))[0] == 1
    assert orc.any(_ray((0, 0, 0), (0, 0, -1)))[0] == 0


def test_icosphere_hit_from_outside():
    """Rays from 5 units away aimed at the centre of a level-4 unit icosphere hit it at
    t in [4, 5 - r_in], r_in = the smallest distance from the centre to a face plane."""
    v, f = scenes.icosphere(4)
    tri = v[f]
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    r_in = np.min(np.abs(np.sum(nrm * tri[:, 0], 1)) / np.linalg.norm(nrm, axis=1))
    sc = scenes.SceneData(v.astype(np.float32), v.astype(np.float32), f.astype(np.uint32),
                          np.zeros(len(f)), MAT, LIGHT)
    rng = np.random.default_rng(3)
    dirs = rng.normal(size=(2000, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.concatenate([5 * dirs, -dirs], 1).astype(np.float32)
    ids, t, _ = oracle.Oracle(sc).closest(rays)
    assert np.all(ids >= 0)
    assert np.all(t >= 4.0 - 1e-5) and np.all(t <= 5.0 - r_in + 1e-5)
    miss = np.concatenate([5 * dirs + 1.5 * np.cross(dirs, [0, 0, 1]) / np.maximum(
        np.linalg.norm(np.cross(dirs, [0, 0, 1]), axis=1, keepdims=True), 1e-9), -dirs], 1).astype(np.float32)
    ids2, _, _ = oracle.Oracle(sc).closest(miss)
    assert np.all(ids2 == -1)


@pytest.mark.gpu
def test_library_gives_the_same_known_answers(ctx):
    from eos_b200 import api
    d = api.DeviceScene(ctx, _point_scene())
    codes, order = d.morton()
    assert sorted(int(c) for c in codes) == sorted(CODES) and list(order) == [0, 2, 1]
    d = api.DeviceScene(ctx, _scene(TRI + TRI + TRI))
    ids, t = api.trace_closest(ctx, d, np.concatenate([_ray((0, 0, 5), (0, 0, -1)), _ray((0, 0, -5), (0, 0, 1)),
                                                       _ray((0, 0, 5), (0, 0, 1)), _ray((2, 0, 5), (0, 0, -1))]))
    assert list(ids) == [2, 2, -1, -1] and t[0] == 5.0 and t[1] == 5.0
    for leg, hit in ((1e-3, False), (1e-2, True)):
        d = api.DeviceScene(ctx, _scene([(0, 0, 0), (leg, 0, 0), (0, leg, 0)]))
        ids, _ = api.trace_closest(ctx, d, _ray((leg / 4, leg / 4, 1), (0, 0, -1)))
        assert (ids[0] == 0) == hit
    d = api.DeviceScene(ctx, _scene([(-1, -1, 3), (1, -1, 3), (0, 1, 3)]))
    occ = api.trace_any(ctx, d, np.concatenate([_ray((0, 0, 0), (0, 0, 1)), _ray((0, 0, 0), (0, 0, -1))]))
    assert list(occ) == [1, 0]
