"""The PLOC builder's tree (eos_b200/csrc/ploc.cu) against the oracle's restatement of its
rules (oracle/ploc.py): every triangle's record position -- the tree's depth-first leaf
order, which the clustering decides merge by merge -- is equal, on scenes that the
builder finishes in its one-block tail alone (at most 1,024 clusters), after a few
per-round launches, and after ~40 of them (205k triangles and the 1.06M-triangle
benchmark scene), and on a grid of equal
triangles where merged areas tie exactly.  A PLOC tree too deep for the refit's walk falls
back to the LBVH."""
import numpy as np
import pytest

from eos_b200 import _lib as L
from eos_b200 import api, scenes
from oracle import ploc as oracle_ploc

pytestmark = pytest.mark.gpu


def _pos_of_id(path):
    """Record position of every triangle id, read from a saved scene file (104-byte header;
    payload: node records, triangle and shading records, then the id -> position map)."""
    raw = np.fromfile(path, np.uint8)
    h = raw[:104].view(np.uint32)
    n_tris, n_nodes = int(h[3]), int(h[4])
    off = 104 + 128 * n_nodes + 96 * max(1, n_tris)
    return raw[off:off + 4 * n_tris].view(np.int32)


@pytest.mark.parametrize("seed,n_spheres,level", [(4, 1, 2), (3, 4, 3), (11, 40, 4)])
def test_ploc_tree_matches_oracle(ctx, tmp_path, seed, n_spheres, level):
    sc = scenes.small_random_scene(seed, n_spheres=n_spheres, level=level, lights=1)
    d = api.DeviceScene(ctx, sc, builder="ploc")
    assert d.info()["builder"] == L.BUILDER_PLOC
    _, order = d.morton()
    lo, hi = oracle_ploc.leaf_boxes(sc.verts, sc.tris, order)
    _, count, position = oracle_ploc.build(lo, hi)
    assert count[-1] == sc.n_tris  # the root holds every leaf
    d.save(tmp_path / "s.eos")
    expect = np.empty(sc.n_tris, np.int64)
    expect[order.astype(np.int64)] = position
    assert np.array_equal(_pos_of_id(tmp_path / "s.eos"), expect)


def _equal_triangles(centres):
    """One right triangle (legs 0.5 along x and y) at each centre."""
    c = np.asarray(centres, np.float64)
    v = (c[:, None, :] + np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0]])).reshape(-1, 3).astype(np.float32)
    mat = [scenes.material((0.5, 0.5, 0.5), 0.2, 16, 0.0)]
    light = np.array([[0, 0, 5, 1, 1, 1]], np.float32)
    nrm = np.tile(np.array([0, 0, 1], np.float32), (len(v), 1))
    return scenes.SceneData(v, nrm, np.arange(len(v)).reshape(-1, 3), np.zeros(len(c)), mat, light)


def test_ploc_ties_match_oracle(ctx, tmp_path):
    xs, ys = np.meshgrid(np.arange(64), np.arange(64))
    sc = _equal_triangles(np.stack([xs.ravel(), ys.ravel(), np.zeros(xs.size)], 1))
    d = api.DeviceScene(ctx, sc, builder="ploc")
    assert d.info()["builder"] == L.BUILDER_PLOC
    _, order = d.morton()
    lo, hi = oracle_ploc.leaf_boxes(sc.verts, sc.tris, order)
    _, _, position = oracle_ploc.build(lo, hi)
    d.save(tmp_path / "g.eos")
    expect = np.empty(sc.n_tris, np.int64)
    expect[order.astype(np.int64)] = position
    assert np.array_equal(_pos_of_id(tmp_path / "g.eos"), expect)


def test_too_deep_ploc_tree_falls_back_to_lbvh(ctx, tmp_path):
    """1,000 triangles at one place: every merged area ties, the clustering makes a chain
    deeper than the refit walks, and the builder makes the LBVH instead -- the same scene
    file, byte for byte but the build time, as asking for the LBVH."""
    sc = _equal_triangles(np.zeros((1000, 3)))
    raw = []
    for builder in ("ploc", "lbvh"):
        d = api.DeviceScene(ctx, sc, builder=builder)
        assert d.info()["builder"] == L.BUILDER_LBVH
        d.save(tmp_path / f"{builder}.eos")
        raw.append((tmp_path / f"{builder}.eos").read_bytes())
    assert raw[0][:56] == raw[1][:56] and raw[0][60:] == raw[1][60:]


def test_ploc_tree_matches_oracle_at_full_size(ctx, tmp_path):
    """The 1,056,768-triangle scene of the 1080p benchmark: every triangle's record position
    equals the restatement's (about 10 s of numpy)."""
    sc = scenes.config2_scene()
    d = api.DeviceScene(ctx, sc, builder="ploc")
    assert d.info()["builder"] == L.BUILDER_PLOC
    _, order = d.morton()
    lo, hi = oracle_ploc.leaf_boxes(sc.verts, sc.tris, order)
    _, count, position = oracle_ploc.build(lo, hi)
    assert count[-1] == sc.n_tris
    d.save(tmp_path / "c2.eos")
    expect = np.empty(sc.n_tris, np.int64)
    expect[order.astype(np.int64)] = position
    assert np.array_equal(_pos_of_id(tmp_path / "c2.eos"), expect)
