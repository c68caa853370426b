"""The reference's own GPU render path on this GPU -- a COMPARISON POINT, test infrastructure.

Loads oracle/_ref/libeosref_gpu.so (the reference's src/kernelInvocations.cu and
src/cudaStructures.cu compiled for sm_100a by oracle/Makefile, with ref_gpu_harness.cu) and
times the reference's DeviceRenderer frame: createCudaScene from the tree its own builder
made (restored from oracle/_ref/<scene>_tree.npz), then rayTrace_MegaKernel, which launches
__rayTrace_MegaKernel (src/kernelInvocations.cu:172-310): one primary ray per pixel and
local Phong over all lights -- no shadow rays, no mirror rays -- on (W/16) x (H/16) blocks
of 16 x 16 threads.  It is not a parity target (its rays and shading differ from the CPU
renderer's, which is the reference this library reproduces).

The reference exits the process on any CUDA error (src/cudaQualifiers.h:35-45), so callers
run this as a process of its own and read one JSON line:

    python -m oracle.ref_gpu --scene config1|config2 [--reps N] [--save IMAGE.npz]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
from ctypes import POINTER, c_float, c_int, c_uint8, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GPU_SO = os.path.join(HERE, "_ref", "libeosref_gpu.so")


def main() -> None:
    sys.path.insert(0, ROOT)
    from oracle import _p, _scene_args, make_ref_tree
    from eos_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="config1", choices=["config1", "config2"])
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--save", default=None, help="write the last frame's RGBA image to this .npz")
    a = ap.parse_args()
    if not os.path.exists(GPU_SO):
        print(json.dumps({"unavailable": "oracle/_ref/libeosref_gpu.so not built (make -C oracle refgpu)"}))
        return
    if a.scene == "config2":
        sc, cam = scenes.config2_scene(), scenes.config2_camera()
    else:
        sc, cam = scenes.config1_scene(), scenes.config1_camera()
    tree = make_ref_tree.load(sc, a.scene)
    if tree is None:
        print(json.dumps({"unavailable": f"oracle/_ref/{a.scene}_tree.npz absent (python -m oracle.make_ref_tree "
                                         f"--scene {a.scene})"}))
        return
    L = ctypes.CDLL(GPU_SO)
    L.eosref_scene_create_from_tree.restype = c_void_p
    L.eosref_scene_create_from_tree.argtypes = [POINTER(c_float), POINTER(c_float), c_int, POINTER(ctypes.c_uint32),
                                                POINTER(ctypes.c_uint32), c_int, POINTER(c_float), c_int,
                                                POINTER(c_float), c_int, POINTER(ctypes.c_int32),
                                                POINTER(ctypes.c_int32), c_int]
    L.eosrefgpu_upload.restype = c_void_p
    L.eosrefgpu_upload.argtypes = [c_void_p]
    L.eosrefgpu_render.restype = c_int
    L.eosrefgpu_render.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_int, POINTER(c_uint8),
                                   POINTER(c_float)]
    perm = np.ascontiguousarray(tree[0], np.int32)
    nodes = np.ascontiguousarray(tree[1], np.int32).reshape(-1, 6)
    h = L.eosref_scene_create_from_tree(*_scene_args(sc), _p(perm, ctypes.c_int32), _p(nodes, ctypes.c_int32),
                                        nodes.shape[0])
    if not h:
        print(json.dumps({"unavailable": "tree file does not match the scene"}))
        return
    d_scene = L.eosrefgpu_upload(h)
    W, H = cam.width, cam.height
    img = np.zeros((H, W, 4), np.uint8)
    ms = c_float(0.0)
    c12 = cam.as_array()
    rc = L.eosrefgpu_render(d_scene, _p(c12, c_float), W, H, a.reps, _p(img, c_uint8), ctypes.byref(ms))
    if rc != 0:
        print(json.dumps({"unavailable": "the reference megakernel's CUDA calls failed"}))
        return
    rays = (W // 16) * 16 * (H // 16) * 16  # one primary ray per thread of its grid
    lit = img[..., :3].max(-1).reshape(-1) > 0  # pixel y * W + x, as threadID_mega (kernelInvocations.cu:28)
    out = {"scene": a.scene, "width": W, "height": H, "reps": a.reps, "ms_per_frame": round(ms.value, 4),
           "primary_rays": rays, "mrays": round(rays / (ms.value * 1e-3) / 1e6, 2), "lit_pixels": int(lit.sum()),
           "kernel": "__rayTrace_MegaKernel (primary rays + local Phong, no shadow / mirror rays)"}
    golden = os.path.join(ROOT, "tests", "golden", "config2_sample.npz")
    if a.scene == "config2" and os.path.exists(golden):
        # The megakernel's rays against the reference CPU renderer's primary hits on the
        # 30,000 sampled pixels: a lit pixel must be one whose primary ray hits something
        # (the two differ only in the half-pixel offset, 0 there and 0.5 in the sample).
        z = np.load(golden)
        hit = z["hits"][:, 0] >= 0
        lp = lit[z["pixels"]]
        out["sample_check"] = {"pixels": int(hit.size), "primary_hits": int(hit.sum()), "lit": int(lp.sum()),
                               "lit_without_hit": int((lp & ~hit).sum()), "hit_and_lit": int((lp & hit).sum())}
    if a.save:
        np.savez_compressed(a.save, rgba=img)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
