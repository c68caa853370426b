"""Test infrastructure: a numpy restatement of the PLOC hierarchy's rules, used only by the
tests to check the GPU builder's tree (eos_b200/csrc/ploc.cu) -- never by the library.

The reference has no counterpart: it builds a CPU SAH tree (src/BVH.cpp:97-111), and the
render results do not depend on the tree.  This restates the published algorithm
(Meister & Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
Construction", IEEE TVCG 2018) with the choices the GPU builder documents, so that the
builder's tree -- seen through the record position of every triangle -- can be compared
exactly:

* clusters start as the leaf boxes in Morton order (box = per-axis min / max of the three
  vertices, float32);
* each cluster's nearest neighbour is the cluster within 16 places whose merged box has the
  smallest surface area dx*dy + dy*dz + dz*dx (float32, evaluated in that order), ties to
  the lower index, 1 (cluster 0) or i - 1 when no area is finite;
* mutual nearest neighbours merge into a new node numbered in creation order (one
  exclusive scan per round), at the lower position; the survivors keep their order;
* a round that merges nothing is followed by a forced round that merges (2k, 2k + 1);
* the root is the last node made; each node's first leaf position in depth-first order
  (left child first) gives the record position of every leaf.
"""
import numpy as np

RADIUS = 16


def _area(al, ah, bl, bh):
    d = (np.maximum(ah, bh) - np.minimum(al, bl)).astype(np.float32)
    dx, dy, dz = d[..., 0], d[..., 1], d[..., 2]
    return (dx * dy + dy * dz) + dz * dx


def leaf_boxes(verts, tris, order):
    """Leaf boxes (lo, hi), float32 [n, 3], in the Morton order `order` (triangle ids)."""
    v = np.asarray(verts, np.float32)[np.asarray(tris, np.int64)[np.asarray(order, np.int64)]]
    return v.min(axis=1), v.max(axis=1)


def build(lo, hi, radius=RADIUS):
    """PLOC over leaf boxes in Morton order.  Returns (child [n-1, 2], count [n-1],
    position [n]): interior nodes in creation order (root n - 2), leaf at Morton position p
    has id n - 1 + p, position[p] = its depth-first record position."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    n = len(lo)
    if n < 2:
        return np.zeros((0, 2), np.int64), np.zeros(0, np.int64), np.zeros(n, np.int64)
    cid = np.arange(n - 1, 2 * n - 1, dtype=np.int64)
    clo, chi = lo.copy(), hi.copy()
    child = np.full((n - 1, 2), -1, np.int64)
    count = np.zeros(n - 1, np.int64)
    node_base, force, rounds = 0, False, 0
    while len(cid) > 1:
        rounds += 1
        assert rounds <= 4 * n + 8
        nc = len(cid)
        i = np.arange(nc)
        if force:
            partner = np.where(i & 1, i - 1, np.where(i + 1 < nc, i + 1, -1))
        else:
            best = np.full(nc, np.inf, np.float32)
            nn = np.where(i == 0, 1, i - 1)
            for d in range(-radius, radius + 1):
                if d == 0:
                    continue
                j = i + d
                ok = (j >= 0) & (j < nc)
                jj = np.clip(j, 0, nc - 1)
                a = _area(clo, chi, clo[jj], chi[jj])
                upd = ok & (a < best)
                best = np.where(upd, a, best)
                nn = np.where(upd, j, nn)
            partner = np.where((nn >= 0) & (nn < nc) & (nn[np.clip(nn, 0, nc - 1)] == i), nn, -1)
        keep = (partner < 0) | (i < partner)
        make = (partner >= 0) & (i < partner)
        pos = np.cumsum(keep) - keep
        mk = np.cumsum(make) - make
        made = int(make.sum())
        if made:
            lo_i, pa = i[make], partner[make]
            k = node_base + mk[make]
            a, b = cid[lo_i], cid[pa]
            child[k, 0], child[k, 1] = a, b
            ca = np.where(a >= n - 1, 1, count[np.clip(a, 0, n - 2)])
            cb = np.where(b >= n - 1, 1, count[np.clip(b, 0, n - 2)])
            count[k] = ca + cb
        new_cid = np.empty(int(keep.sum()), np.int64)
        new_lo = np.empty((len(new_cid), 3), np.float32)
        new_hi = np.empty((len(new_cid), 3), np.float32)
        solo = keep & (partner < 0)
        new_cid[pos[solo]] = cid[solo]
        new_lo[pos[solo]] = clo[solo]
        new_hi[pos[solo]] = chi[solo]
        if made:
            new_cid[pos[make]] = node_base + mk[make]
            new_lo[pos[make]] = np.minimum(clo[make], clo[partner[make]])
            new_hi[pos[make]] = np.maximum(chi[make], chi[partner[make]])
        node_base += made
        cid, clo, chi = new_cid, new_lo, new_hi
        force = made == 0 and not force
    assert node_base == n - 1
    first = np.zeros(2 * n - 1, np.int64)
    for k in range(n - 2, -1, -1):  # parents are made after their children
        a, b = child[k]
        first[a] = first[k]
        first[b] = first[k] + (1 if a >= n - 1 else count[a])
    return child, count, first[n - 1:]
