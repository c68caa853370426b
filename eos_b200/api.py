"""Python view of the C ABI: context, resident scenes, render / batch / backward / queries.

Device buffers are torch CUDA tensors (torch is used for device memory only); host
buffers are numpy arrays, which the library stages through its own device memory.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from ctypes import byref, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .scenes import CameraData, SceneData, pad_materials


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(c_void_p)


def camera_struct(cam: CameraData) -> L.Camera:
    c = L.Camera()
    for k in range(3):
        c.position[k] = float(cam.position[k])
        c.view[k] = float(cam.view[k])
        c.right[k] = float(cam.right[k])
        c.up[k] = float(cam.up[k])
    c.width = int(cam.width)
    c.height = int(cam.height)
    return c


def tree_nodes(trace_depth: int) -> int:
    """Nodes of a tree-form path record: 2^(trace_depth + 1) - 1 (EOS_TREE_NODES)."""
    return (1 << (int(trace_depth) + 1)) - 1


def params_struct(trace_depth=1, pixel_offset=0.5, spp=1, jitter_seed=0, mode="plain", block_size=0,
                  queue_chunk=0, stack_depth=0, stage_timing=False, rows=None,
                  tree_records=False, aa_grid=False) -> L.RenderParams:
    p = L.RenderParams()
    p.trace_depth = int(trace_depth)
    p.pixel_offset = float(pixel_offset)
    p.spp = int(spp)
    p.jitter_seed = int(jitter_seed)
    p.mode = L.MODE_WAVEFRONT if mode == "wavefront" else L.MODE_PLAIN
    p.block_size = int(block_size)
    p.queue_chunk = int(queue_chunk)
    p.stack_depth = int(stack_depth)
    p.flags = ((L.FLAG_STAGE_TIMING if stage_timing else 0) | (L.FLAG_TREE_RECORDS if tree_records else 0)
               | (L.FLAG_AA_GRID if aa_grid else 0))
    if rows is not None:
        p.row_begin, p.row_end = int(rows[0]), int(rows[1])
    return p


def stats_dict(st: L.Stats) -> dict:
    d = {f: getattr(st, f) for f, _ in L.Stats._fields_ if f != "stage_ms"}
    d["stage_ms"] = [float(v) for v in st.stage_ms]
    return d


class Context:
    def __init__(self, device: int = 0):
        self.lib = L.load()
        self._scenes = weakref.WeakSet()  # scenes on this context, destroyed before it
        h = c_void_p()
        L.check(self.lib.eos_ctx_create(device, byref(h)), "eos_ctx_create")
        self.h = h
        self.device = device

    def close(self):
        """Destroy the context and, first, every scene still open on it (a scene's
        destroy reaches its context's stream)."""
        if getattr(self, "h", None):
            for sc in list(getattr(self, "_scenes", ())):
                sc.close()
            self.lib.eos_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        L.check(self.lib.eos_ctx_set_stream(self.h, c_void_p(stream_handle) if stream_handle else None),
                "eos_ctx_set_stream")

    def synchronize(self):
        """Waits for the context (the copies of asynchronous batches included); raises the first
        device error of the asynchronous batches since the last call and returns their stats
        dicts in issue order."""
        pending, self._async_stats = getattr(self, "_async_stats", []), []
        L.check(self.lib.eos_ctx_synchronize(self.h), "eos_ctx_synchronize")
        return [stats_dict(st) for st in pending]

    def set_limits(self, queue_entries: int = 0, work_budget: int = 0, small_stack: bool = False):
        """Test limits of the wavefront kernels (eos_ctx_set_limits); no arguments clears them."""
        lim = L.Limits(int(queue_entries), int(work_budget), 1 if small_stack else 0)
        L.check(self.lib.eos_ctx_set_limits(self.h, byref(lim)), "eos_ctx_set_limits")


def materials_array(mats):
    """Material rows in the C layout (eos_material, 10 floats): numpy rows of 8 or 10, or a
    torch tensor (rows of 8 are padded with transparency 0, refractive index 1)."""
    if hasattr(mats, "data_ptr"):
        import torch
        m = mats.float().reshape(mats.shape[0], -1)
        if m.shape[1] == 8:
            pad = torch.tensor([0.0, 1.0], device=m.device).expand(m.shape[0], 2)
            m = torch.cat([m, pad], 1)
        return m.contiguous()
    return pad_materials(mats)


class DeviceScene:
    """A scene resident in HBM with its LBVH (eos_scene_create)."""

    def __init__(self, ctx: Context, scene: SceneData, leaf_size: int = 0, inputs_on_device: bool = False,
                 layout: str | int = 0, width: int = 0, builder: str | int = 0):
        """leaf_size / layout / width / builder 0 take the context's tuned values for this scene
        size (without a table: PLOC hierarchy, 4-wide nodes, SAH collapse, leaves of <= 8)."""
        self.ctx = ctx
        self.scene = scene
        self.lib = ctx.lib
        bp = L.BuildParams()
        bp.leaf_size = leaf_size
        bp.layout = {"sah": L.LAYOUT_SAH, "fixed": L.LAYOUT_FIXED}.get(layout, layout) if layout else 0
        bp.width = int(width)
        bp.builder = {"lbvh": L.BUILDER_LBVH, "ploc": L.BUILDER_PLOC}.get(builder, builder) if builder else 0
        arrs = [scene.verts, scene.normals, scene.tris, scene.tri_obj]
        if inputs_on_device:
            import torch
            arrs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]
        mats = materials_array(scene.materials)
        lights = np.ascontiguousarray(scene.lights, np.float32)
        h = c_void_p()
        code = self.lib.eos_scene_create(ctx.h, _ptr(arrs[0]), _ptr(arrs[1]), scene.verts.shape[0], _ptr(arrs[2]),
                                         _ptr(arrs[3]), scene.n_tris, _ptr(mats), mats.shape[0], _ptr(lights),
                                         lights.shape[0], byref(bp), byref(h))
        L.check(code, "eos_scene_create")
        self.h = h
        ctx._scenes.add(self)
        if scene.ambient_index != 1.0:
            self.set_ambient_index(scene.ambient_index)

    def close(self):
        if getattr(self, "h", None):
            self.lib.eos_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        i = L.SceneInfo()
        L.check(self.lib.eos_scene_get_info(self.h, byref(i)), "eos_scene_get_info")
        return {f: getattr(i, f) for f, _ in L.SceneInfo._fields_}

    def morton(self):
        n = self.scene.n_tris
        codes = np.zeros(n, np.uint32)
        order = np.zeros(n, np.uint32)
        L.check(self.lib.eos_scene_get_morton(self.h, _ptr(codes), _ptr(order)), "eos_scene_get_morton")
        return codes, order

    def set_materials(self, mats):
        m = materials_array(mats)
        L.check(self.lib.eos_scene_set_materials(self.h, _ptr(m), int(m.shape[0])), "eos_scene_set_materials")

    def set_ambient_index(self, refractive_index: float):
        L.check(self.lib.eos_scene_set_ambient_index(self.h, float(refractive_index)), "eos_scene_set_ambient_index")

    def set_lights(self, lights):
        l = lights if hasattr(lights, "data_ptr") else np.ascontiguousarray(lights, np.float32).reshape(-1, 6)
        L.check(self.lib.eos_scene_set_lights(self.h, _ptr(l), int(l.shape[0])), "eos_scene_set_lights")

    def save(self, path):
        """Write the built scene to a file (eos_scene_save)."""
        L.check(self.lib.eos_scene_save(self.h, os.fsencode(path)), "eos_scene_save")

    @classmethod
    def load(cls, ctx: Context, path, scene: SceneData | None = None) -> "DeviceScene":
        """A scene read from a file of eos_scene_save, with no build (eos_scene_load).
        scene: the SceneData it was made from, where the caller has it (render_backward
        and morton read its sizes)."""
        self = cls.__new__(cls)
        self.ctx, self.lib, self.scene = ctx, ctx.lib, scene
        h = c_void_p()
        L.check(self.lib.eos_scene_load(ctx.h, os.fsencode(path), byref(h)), "eos_scene_load")
        self.h = h
        ctx._scenes.add(self)
        return self


class InstancedScene(DeviceScene):
    """A two-level scene (eos_scene_create_instanced): placements of mesh scenes.

    meshes: DeviceScene objects used as geometry (kept alive by this object);
    instances: (mesh index, 3x4 world-from-object transform, material base) per instance;
    materials [K, 10] / lights [L, 6] of the whole scene.  Hit ids are global: instance k's
    triangles follow those of instances 0..k-1."""

    def __init__(self, ctx: Context, meshes: list, instances: list, materials, lights, ambient_index: float = 1.0):
        self.ctx = ctx
        self.lib = ctx.lib
        self.meshes = list(meshes)
        arr = (L.Instance * len(instances))()
        for i, (mi, M, base) in enumerate(instances):
            arr[i].mesh = self.meshes[mi].h
            for k, v in enumerate(np.asarray(M, np.float64).reshape(3, 4).reshape(-1)):
                arr[i].transform[k] = float(v)
            arr[i].material_base = int(base)
        mats = materials_array(materials)
        lts = np.ascontiguousarray(lights, np.float32).reshape(-1, 6)
        h = c_void_p()
        L.check(self.lib.eos_scene_create_instanced(ctx.h, arr, len(instances), _ptr(mats), mats.shape[0], _ptr(lts),
                                                    lts.shape[0], byref(h)), "eos_scene_create_instanced")
        self.h = h
        ctx._scenes.add(self)
        self.n_tris = sum(self.meshes[mi].scene.n_tris for mi, _, _ in instances)
        self.scene = None
        if ambient_index != 1.0:
            self.set_ambient_index(ambient_index)


def _alloc(shape, dtype, device: bool):
    if device:
        import torch
        tmap = {np.float32: torch.float32, np.uint8: torch.uint8, np.int32: torch.int32}
        return torch.empty(shape, dtype=tmap[dtype], device="cuda")
    return np.empty(shape, dtype)


def render(ctx: Context, scene: DeviceScene, cam: CameraData, trace_depth: int, pixel_offset: float = 0.5,
           spp: int = 1, jitter_seed: int = 0, mode: str = "plain", outputs=("rgb",), device: bool = True,
           out: dict | None = None, **tuning) -> dict:
    """Render one frame; returns the requested outputs plus 'stats'.

    outputs: any of 'rgb' [H*W,3] f32, 'rgba8' [H,W,4] u8, 'hit' [H*W*spp] i32,
    'paths' [H*W*spp, 16] i32 (8 hit ids then 8 shadow masks per path; with
    tree_records=True in `tuning`, [H*W*spp, tree_nodes(trace_depth), 2]: hit id and shadow
    mask per ray-tree node).  rows=(r0, r1) in `tuning` renders image rows [r0, r1) only
    (split-frame); H is then r1 - r0.
    """
    rows = tuning.get("rows")
    H = (rows[1] - rows[0]) if rows is not None else cam.height
    npx = cam.width * H
    res = dict(out or {})
    shapes = {"rgb": ((npx, 3), np.float32), "rgba8": ((H, cam.width, 4), np.uint8),
              "hit": ((npx * spp,), np.int32),
              "paths": ((npx * spp, tree_nodes(trace_depth), 2) if tuning.get("tree_records") else (npx * spp, 16),
                        np.int32)}
    for k in outputs:
        if k not in res:
            res[k] = _alloc(shapes[k][0], shapes[k][1], device)
    st = L.Stats()
    c = camera_struct(cam)
    p = params_struct(trace_depth, pixel_offset, spp, jitter_seed, mode, **tuning)
    code = ctx.lib.eos_render(ctx.h, scene.h, byref(c), byref(p), _ptr(res.get("rgb")), _ptr(res.get("rgba8")),
                              _ptr(res.get("hit")), _ptr(res.get("paths")), byref(st))
    L.check(code, "eos_render")
    res["stats"] = stats_dict(st)
    return res


@dataclass
class BatchJob:
    scene: DeviceScene
    camera: CameraData
    trace_depth: int = 1
    pixel_offset: float = 0.5
    spp: int = 1
    jitter_seed: int = 0
    rows: tuple | None = None  # image rows [r0, r1) only


def make_batch_outputs(jobs: list[BatchJob], outputs=("rgb",), tree_records: bool = False):
    outs = []
    for j in jobs:
        H = (j.rows[1] - j.rows[0]) if j.rows is not None else j.camera.height
        npx = j.camera.width * H
        o = {}
        if "rgb" in outputs:
            o["rgb"] = _alloc((npx, 3), np.float32, True)
        if "rgba8" in outputs:
            o["rgba8"] = _alloc((H, j.camera.width, 4), np.uint8, True)
        if "paths" in outputs:
            shape = (npx * j.spp, tree_nodes(j.trace_depth), 2) if tree_records else (npx * j.spp, 16)
            o["paths"] = _alloc(shape, np.int32, True)
        outs.append(o)
    return outs


def render_batch(ctx: Context, jobs: list[BatchJob], outs: list[dict], async_outputs: bool = False,
                 **tuning) -> dict | None:
    """All jobs through one wavefront pass (graph-captured); outputs are device tensors or host
    arrays (host outputs are filled when the call returns).  async_outputs=True
    (EOS_FLAG_ASYNC): returns None once the batch is queued; host outputs (pinned) are
    filled, and the call's stats returned, by ctx.synchronize()."""
    arr = (L.Job * len(jobs))()
    for i, (j, o) in enumerate(zip(jobs, outs)):
        arr[i].scene = j.scene.h
        arr[i].camera = camera_struct(j.camera)
        arr[i].trace_depth = j.trace_depth
        arr[i].pixel_offset = j.pixel_offset
        arr[i].spp = j.spp
        arr[i].jitter_seed = j.jitter_seed
        arr[i].rgb_out = _ptr(o.get("rgb"))
        arr[i].rgba8_out = _ptr(o.get("rgba8"))
        arr[i].paths_out = _ptr(o.get("paths"))
        if j.rows is not None:
            arr[i].row_begin, arr[i].row_end = int(j.rows[0]), int(j.rows[1])
    p = params_struct(mode="wavefront", **tuning)
    if async_outputs:
        p.flags |= L.FLAG_ASYNC
    st = L.Stats()
    L.check(ctx.lib.eos_render_batch(ctx.h, arr, len(jobs), byref(p), byref(st)), "eos_render_batch")
    if async_outputs:
        if not hasattr(ctx, "_async_stats"):
            ctx._async_stats = []
        ctx._async_stats.append(st)  # filled by eos_ctx_synchronize: kept alive until then
        return None
    return stats_dict(st)


def render_backward(ctx: Context, scene: DeviceScene, cams: list[CameraData], trace_depth: int, paths, d_rgb,
                    pixel_offset: float = 0.5, device: bool = True, spp: int = 1, jitter_seed: int = 0,
                    rows=None, tree_records: bool = False, aa_grid: bool = False):
    """Adjoint of the shading: returns (grad_materials [K,7], grad_lights [L,6]).  paths come
    from the forward render with the same spp / jitter_seed / pixel_offset (and row band
    `rows`, whose gradients are that band's share of the frame's)."""
    arr = (L.Camera * len(cams))(*[camera_struct(c) for c in cams])
    p = params_struct(trace_depth, pixel_offset, spp, jitter_seed, rows=rows, tree_records=tree_records,
                      aa_grid=aa_grid)
    info = scene.info()
    K = info["n_objects"]
    NL = max(1, info["n_lights"])
    gm = _alloc((K, 7), np.float32, device)
    gl = _alloc((NL, 6), np.float32, device)
    g = L.Grads()
    g.materials = _ptr(gm).value
    g.lights = _ptr(gl).value
    code = ctx.lib.eos_render_backward(ctx.h, scene.h, arr, len(cams), byref(p), _ptr(paths), _ptr(d_rgb), byref(g))
    L.check(code, "eos_render_backward")
    return gm, gl


def trace_closest(ctx: Context, scene: DeviceScene, rays: np.ndarray):
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
    n = r.shape[0]
    ids = np.zeros(n, np.int32)
    ts = np.zeros(n, np.float32)
    L.check(ctx.lib.eos_trace_closest(ctx.h, scene.h, _ptr(r), n, _ptr(ids), _ptr(ts)), "eos_trace_closest")
    return ids, ts


def trace_any(ctx: Context, scene: DeviceScene, rays: np.ndarray):
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
    n = r.shape[0]
    occ = np.zeros(n, np.uint8)
    L.check(ctx.lib.eos_trace_any(ctx.h, scene.h, _ptr(r), n, _ptr(occ)), "eos_trace_any")
    return occ
