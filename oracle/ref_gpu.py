"""The reference's own GPU render path on this GPU -- a COMPARISON POINT, test infrastructure.

Loads oracle/_ref/libeosref_gpu.so (the reference's src/kernelInvocations.cu and
src/cudaStructures.cu compiled for sm_100a by oracle/Makefile, with ref_gpu_harness.cu) and
times the reference's DeviceRenderer frame: createCudaScene from the tree its own builder
made (restored from oracle/_ref/<scene>_tree.npz, or built here for the small transformed
scene), then rayTrace_MegaKernel, which launches __rayTrace_MegaKernel
(src/kernelInvocations.cu:172-310): one primary ray per pixel and local Phong over all
lights -- no shadow rays, no mirror rays -- on (W/16) x (H/16) blocks of 16 x 16 threads.
Its shading is not the CPU renderer's (the reference this library reproduces), so it is
not a parity target for colours; megakernel_colours restates that shading for a given set
of hits, so that its image checks which triangle each primary ray hit.

The reference exits the process on any CUDA error (src/cudaQualifiers.h:35-45), so callers
run this as a process of its own and read one JSON line:

    python -m oracle.ref_gpu --scene config1|config2|transformed [--reps N] [--save IMAGE.npz]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
from ctypes import POINTER, c_float, c_int, c_uint8, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GPU_SO = os.path.join(HERE, "_ref", "libeosref_gpu.so")


def transformed_case(seed: int = 7, size: int = 256):
    """A two-level scene (scenes.InstancedData) and camera that the reference's GPU path
    renders correctly, for checking placements against it.

    Placements are translations and axis scales, non-uniform and mirrored ones among them:
    the reference bounds a transformed triangle by transforming its local box's two
    corners only (Box::transformBoundingBox, src/Box.cu:84-135), which holds the triangle
    under those placements and not under rotations.  The ground is a slightly warped quad:
    the kernel's box test asks tmin < tmax (src/kernelInvocations.h:60-73), which a box of
    zero thickness never passes, so it cannot see a triangle lying in an axis plane.  The
    lights are on the camera's side of the origin, so that the megakernel's specular term
    of a ray that hits nothing is 0 (src/kernelInvocations.cu:246-300 shades misses with a
    zero point and normal)."""
    sys.path.insert(0, ROOT)
    from eos_b200 import scenes
    rng = scenes.rng_for(seed)
    grey = [scenes.material((0.5, 0.5, 0.5), 0.2, 16, 0.0)]
    v, f = scenes.icosphere(2)
    qv, qn, qf = scenes.ground_quad(4.0, 0.0)
    qv[:, 1] = (0.0, 0.15, 0.05, 0.2)  # warped: no triangle lies in an axis plane
    qn = np.cross(qv[qf[:, 1]] - qv[qf[:, 0]], qv[qf[:, 2]] - qv[qf[:, 0]])
    qn = np.repeat(qn / np.linalg.norm(qn, axis=1, keepdims=True), 3, axis=0)
    qv, qf = qv[qf.reshape(-1)], np.arange(6).reshape(2, 3)  # flat-shaded: vertices per triangle
    cv, cn, cf = scenes.foliage_cluster(300, rng, radius=1.0)
    meshes = [scenes.SceneData(v, v, f, np.zeros(len(f)), grey, np.zeros((0, 6))),
              scenes.SceneData(qv, qn, qf, np.zeros(len(qf)), grey, np.zeros((0, 6))),
              scenes.SceneData(cv, cn, cf, np.zeros(len(cf)), grey, np.zeros((0, 6)))]

    def place(scale, t):
        M = np.zeros((3, 4))
        M[:, :3] = np.diag(scale)
        M[:, 3] = t
        return M

    instances = [(1, place((1.5, 1.0, 1.5), (0.0, -2.5, 0.0)), 0)]
    mats = [scenes.material(rng.uniform(0, 1, 3), 0.3, 8, 0.0)]
    for k in range(1, 12):
        s = rng.uniform(0.4, 1.2) * np.ones(3)
        if k == 2:
            s *= (1.0, 0.5, 1.5)  # non-uniform
        if k == 3:
            s *= (-1.0, 1.0, 1.0)  # mirrored
        if k == 5:
            s *= (1.3, -0.7, 1.0)  # non-uniform and mirrored
        t = rng.uniform([-3, -1.5, -3], [3, 1.5, 3])
        instances.append((0 if k % 2 else 2, place(s, t), k))
        mats.append(scenes.material(rng.uniform(0, 1, 3), rng.uniform(0, 0.5), float(rng.integers(4, 64)), 0.0))
    lights = [[4.0, 7.0, 8.0, 1.0, 1.0, 1.0], [-3.0, 6.0, 7.0, 0.8, 0.8, 0.8]]
    d = scenes.InstancedData(meshes, instances, np.array(mats), np.array(lights), f"transformed{seed}")
    cam = scenes.look_at((1.0, 3.0, 9.0), (0.0, -0.5, 0.0), 55.0, size, size)
    return d, cam


def object_space_arrays(d):
    """The reference's per-triangle form of a two-level scene: object-space vertices and
    normals, triangles in global-id order (instance k's after instances 0..k-1), material
    ids, each triangle's transformation index and the transformations [K, 12]."""
    V, N, F, O, X = [], [], [], [], []
    nv = 0
    for k, (m, M, base) in enumerate(d.instances):
        sc = d.meshes[m]
        V.append(sc.verts)
        N.append(sc.normals)
        F.append(sc.tris.astype(np.int64) + nv)
        O.append(sc.tri_obj.astype(np.int64) + base)
        X.append(np.full(sc.n_tris, k, np.int32))
        nv += sc.verts.shape[0]
    xf = np.array([np.asarray(M, np.float32).reshape(12) for _, M, _ in d.instances], np.float32)
    return (np.ascontiguousarray(np.concatenate(V), np.float32), np.ascontiguousarray(np.concatenate(N), np.float32),
            np.ascontiguousarray(np.concatenate(F), np.uint32), np.ascontiguousarray(np.concatenate(O), np.uint32),
            np.ascontiguousarray(np.concatenate(X), np.int32), xf)


def megakernel_colours(verts, normals, tris, tri_mat, tri_xf, xforms, materials, lights, cam, hits):
    """RGBA8 [H, W, 4] that __rayTrace_MegaKernel writes (src/kernelInvocations.cu:190-310)
    for the given primary hits [H * W] (triangle ids, -1 for none), in float64: the ray
    normalize(((2x - W) / W) right + ((2y - H) / H) up + view), moved into the triangle's
    object space by the inverse of its transformation; barycentrics from the reference's
    Moller-Trumbore; the interpolated unit normal times the inverse transpose, not
    renormalised; per light max(0, L.N) kd lc + max(0, V.R)^shininess lc ks; saturated and
    scaled by 255 with truncation.  A pixel with no hit is black."""
    W, H = cam.width, cam.height
    x, y = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    c = [np.asarray(a, np.float64) for a in (cam.position, cam.view, cam.right, cam.up)]
    d = (((2.0 * x - W) / W).reshape(-1, 1) * c[2] + ((2.0 * y - H) / H).reshape(-1, 1) * c[3] + c[1])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    out = np.zeros((H * W, 4), np.uint8)
    out[:, 3] = 255
    hit = np.asarray(hits).reshape(-1)
    sel = np.nonzero(hit >= 0)[0]
    if sel.size == 0:
        return out.reshape(H, W, 4)
    tri = hit[sel]
    M4 = np.zeros((len(xforms), 4, 4))
    M4[:, :3, :] = np.asarray(xforms, np.float64).reshape(-1, 3, 4)
    M4[:, 3, 3] = 1.0
    inv = np.linalg.inv(M4)
    inv_t = np.linalg.inv(np.transpose(M4, (0, 2, 1)))
    k = tri_xf[tri]
    o = np.broadcast_to(c[0], (sel.size, 3))
    o_l = np.einsum("nij,nj->ni", inv[k][:, :3, :3], o) + inv[k][:, :3, 3]
    d_l = np.einsum("nij,nj->ni", inv[k][:, :3, :3], d[sel])
    tv = tris[tri].astype(np.int64)
    v1, v2, v3 = (verts[tv[:, j]].astype(np.float64) for j in range(3))
    e1, e2 = v2 - v1, v3 - v1
    P = np.cross(d_l, e2)
    det = (e1 * P).sum(1)
    T = o_l - v1
    Q = np.cross(T, e1)
    t = (e2 * Q).sum(1) / det
    u = (T * P).sum(1) / det
    v = (d_l * Q).sum(1) / det
    n1, n2, n3 = (normals[tv[:, j]].astype(np.float64) for j in range(3))
    n = n1 * (1.0 - u - v)[:, None] + n2 * u[:, None] + n3 * v[:, None]
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    N = np.einsum("nij,nj->ni", inv_t[k][:, :3, :3], n)  # w of the product never enters a dot below
    Pw = o + t[:, None] * d[sel]
    mat = np.asarray(materials, np.float64)[tri_mat[tri]]
    kd, ks, sh = mat[:, 0:3], mat[:, 3:6], mat[:, 6]
    V = c[0] - Pw
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    col = np.zeros((sel.size, 3))
    for light in np.asarray(lights, np.float64).reshape(-1, 6):
        L = light[:3] - Pw
        L /= np.linalg.norm(L, axis=1, keepdims=True)
        ln = (L * N).sum(1)
        R = -L + 2.0 * ln[:, None] * N
        col += np.maximum(0.0, ln)[:, None] * kd * light[3:6]
        col += (np.maximum(0.0, (V * R).sum(1)) ** sh)[:, None] * light[3:6] * ks
    out[sel, :3] = (np.clip(col, 0.0, 1.0) * 255.0).astype(np.uint8)
    return out.reshape(H, W, 4)


def _lib():
    L = ctypes.CDLL(GPU_SO)
    L.eosref_scene_create_from_tree.restype = c_void_p
    L.eosref_scene_create_from_tree.argtypes = [POINTER(c_float), POINTER(c_float), c_int, POINTER(c_uint32),
                                                POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                                POINTER(c_float), c_int, POINTER(ctypes.c_int32),
                                                POINTER(ctypes.c_int32), c_int]
    L.eosref_scene_create_transformed.restype = c_void_p
    L.eosref_scene_create_transformed.argtypes = [POINTER(c_float), POINTER(c_float), POINTER(c_uint32),
                                                  POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                                  POINTER(c_float), c_int, POINTER(ctypes.c_int32),
                                                  POINTER(c_float), c_int, c_int]
    L.eosrefgpu_upload.restype = c_void_p
    L.eosrefgpu_upload.argtypes = [c_void_p]
    L.eosrefgpu_render.restype = c_int
    L.eosrefgpu_render.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_int, POINTER(c_uint8),
                                   POINTER(c_float)]
    return L


def main() -> None:
    sys.path.insert(0, ROOT)
    from oracle import _p, _scene_args, make_ref_tree
    from eos_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="config1", choices=["config1", "config2", "transformed"])
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--save", default=None, help="write the last frame's RGBA image to this .npz")
    a = ap.parse_args()
    if not os.path.exists(GPU_SO):
        print(json.dumps({"unavailable": "oracle/_ref/libeosref_gpu.so not built (make -C oracle refgpu)"}))
        return
    L = _lib()
    if a.scene == "transformed":
        d, cam = transformed_case()
        verts, normals, tris, tri_mat, tri_xf, xf = object_space_arrays(d)
        mats = np.ascontiguousarray(d.materials, np.float32)
        lts = np.ascontiguousarray(d.lights, np.float32)
        h = L.eosref_scene_create_transformed(_p(verts, c_float), _p(normals, c_float), _p(tris, c_uint32),
                                              _p(tri_mat, c_uint32), tris.shape[0], _p(mats, c_float), mats.shape[0],
                                              _p(lts, c_float), lts.shape[0], _p(tri_xf, ctypes.c_int32),
                                              _p(xf, c_float), xf.shape[0], 1)
    else:
        if a.scene == "config2":
            sc, cam = scenes.config2_scene(), scenes.config2_camera()
        else:
            sc, cam = scenes.config1_scene(), scenes.config1_camera()
        tree = make_ref_tree.load(sc, a.scene)
        if tree is None:
            print(json.dumps({"unavailable": f"oracle/_ref/{a.scene}_tree.npz absent (python -m oracle.make_ref_tree "
                                             f"--scene {a.scene})"}))
            return
        perm = np.ascontiguousarray(tree[0], np.int32)
        nodes = np.ascontiguousarray(tree[1], np.int32).reshape(-1, 6)
        h = L.eosref_scene_create_from_tree(*_scene_args(sc), _p(perm, ctypes.c_int32), _p(nodes, ctypes.c_int32),
                                            nodes.shape[0])
    if not h:
        print(json.dumps({"unavailable": "the reference scene could not be made (tree file or arrays invalid)"}))
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
