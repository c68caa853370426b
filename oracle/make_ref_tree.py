"""Builds the reference's own BVH for the 1.06M-triangle benchmark scene (or the
20,482-triangle config-1 scene) once and saves it under oracle/_ref/ -- TEST
INFRASTRUCTURE (the CPU baseline, the reference parity checks and the reference's GPU
comparison point restore it instead of building it again).

The reference's builder (src/BVH.cpp:97-111, 549-606) runs single-threaded here (its SAH
sweep races under OpenMP, src/BVH.cpp:454-480); on the 1,056,768-triangle scene it takes
several minutes, so the tree is built once, exported with eosref_tree_export (the surface
order after the build's sorts and the flat node buffer's topology) and restored by
eosref_scene_create_from_tree, which recomputes every box with the builder's own
BVH::computeBoxWithSurfaces.  The file lives beside the compiled reference in
oracle/_ref/ (ignored by git, shipped with the built libraries).

    python -m oracle.make_ref_tree [--scene config1|config2|config5] [--force]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
def tree_file(name: str = "config2") -> str:
    return os.path.join(HERE, "_ref", f"{name}_tree.npz")


def scene_digest(sc) -> str:
    """Hash of the scene arrays the tree was built for."""
    h = hashlib.sha256()
    for a in (sc.verts, sc.normals, sc.tris, sc.tri_obj):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def load(sc, name: str = "config2"):
    """(perm, nodes) of the saved tree when it was built for scene sc, else None."""
    path = tree_file(name)
    if not os.path.exists(path):
        return None
    z = np.load(path)
    if str(z["digest"]) != scene_digest(sc):
        return None
    return z["perm"], z["nodes"]


def main() -> None:
    sys.path.insert(0, ROOT)
    import oracle
    from eos_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--scene", default="config2", choices=["config1", "config2", "config5"])
    a = ap.parse_args()
    sc = {"config1": scenes.config1_scene, "config2": scenes.config2_scene, "config5": scenes.config5_scene}[a.scene]()
    path = tree_file(a.scene)
    if not a.force and load(sc, a.scene) is not None:
        print(f"{path}: up to date")
        return
    t0 = time.time()
    r = oracle.RefRenderer(sc, build_threads=1)
    perm, nodes = r.export_tree()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, perm=perm, nodes=nodes, digest=np.array(scene_digest(sc)),
                        build_seconds=np.array(r.build_seconds))
    print(f"{path}: {r.n_nodes} nodes, max leaf {r.max_leaf}, build {r.build_seconds:.1f} s "
          f"({time.time() - t0:.1f} s in all)")


if __name__ == "__main__":
    main()
