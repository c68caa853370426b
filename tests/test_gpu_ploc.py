"""The PLOC builder's tree (eos_b200/csrc/ploc.cu) against the oracle's restatement of its
rules (oracle/ploc.py): every triangle's record position -- the tree's depth-first leaf
order, which the clustering decides merge by merge -- is equal, on scenes that the
builder finishes in its one-block tail alone (at most 1,024 clusters), after a few
per-round launches, and after ~40 of them (205k triangles)."""
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
