"""Multi-GPU plumbing: one process per GPU.

Two ways to spread rendering over ranks, both with the scene replicated per GPU as the
reference does (src/MultiDeviceRenderer.cu:59-81):
* views sharded across ranks, no data-path collective (views are independent);
* split-frame: one frame cut into horizontal bands, one per rank, each rendered with a
  row band (eos_render_params.row_begin / row_end) and gathered to every rank with one
  all-gather -- the reference's MultiDeviceRenderer split (src/MultiDeviceRenderer.cu:
  119-200) across processes.
The adjoint has one real exchange step: the parameter-gradient vector (per-object
kd/ks/log-shininess, per-light colour/position) is summed over ranks with one all-reduce.
"""
from __future__ import annotations

import numpy as np


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (balances uneven view sizes)."""
    return list(items)[rank::world]


def shard_indices(n: int, rank: int, world: int) -> np.ndarray:
    return np.arange(rank, n, world)


def band(height: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [r0, r1) of band `rank` out of `world`: height // world rows each, the last
    band takes the remainder (the reference drops it, src/MultiDeviceRenderer.cu:128)."""
    per = height // world
    r0 = rank * per
    r1 = height if rank == world - 1 else r0 + per
    return r0, r1


def gather_bands(mine, height: int, group=None):
    """All-gather of every rank's band (a [rows, W, C] tensor or array) into the whole
    [height, W, C] frame on every rank; bands are padded to equal size for the collective."""
    import torch
    import torch.distributed as dist
    as_np = not hasattr(mine, "data_ptr")
    t = torch.as_tensor(np.asarray(mine)) if as_np else mine
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if world == 1:
        return mine
    per = height // world
    tallest = height - per * (world - 1)
    pad = torch.zeros((tallest,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    full = torch.cat([p[: band(height, r, world)[1] - band(height, r, world)[0]] for r, p in enumerate(parts)])
    return full.numpy() if as_np else full


def render_split_frame(ctx, dscene, cam, trace_depth, rank: int, world: int, pixel_offset=0.5, mode="plain"):
    """This rank's band of one frame (RGBA8 on the device), then the whole frame on every
    rank.  Bit-identical to rendering the frame on one GPU."""
    from . import api
    r0, r1 = band(cam.height, rank, world)
    out = api.render(ctx, dscene, cam, trace_depth, pixel_offset=pixel_offset, mode=mode, outputs=("rgba8",),
                     rows=(r0, r1))
    return gather_bands(out["rgba8"], cam.height)


def allreduce_grads(grad_mat, grad_light, group=None):
    """Sums the gradient arrays over all ranks in place (torch tensors or numpy arrays)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return grad_mat, grad_light
    as_np = not hasattr(grad_mat, "data_ptr")
    gm = torch.as_tensor(np.asarray(grad_mat)) if as_np else grad_mat
    gl = torch.as_tensor(np.asarray(grad_light)) if as_np else grad_light
    flat = torch.cat([gm.reshape(-1), gl.reshape(-1)])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    gm_out = flat[: gm.numel()].reshape(gm.shape)
    gl_out = flat[gm.numel():].reshape(gl.shape)
    if as_np:
        return gm_out.numpy(), gl_out.numpy()
    gm.copy_(gm_out)
    gl.copy_(gl_out)
    return gm, gl


def render_backward_sharded(ctx, dscene, cams, trace_depth, d_rgb_fn, rank: int, world: int, pixel_offset=0.5):
    """Forward + adjoint over this rank's views, gradients summed over all ranks.

    d_rgb_fn(view_index, rgb) returns dL/drgb for that view (device tensor).
    """
    import torch

    from . import api
    mine = shard_indices(len(cams), rank, world)
    info = dscene.info()
    K = info["n_objects"]
    NL = max(1, info["n_lights"])
    gm = torch.zeros((K, 7), device="cuda")
    gl = torch.zeros((NL, 6), device="cuda")
    for v in mine:
        r = api.render(ctx, dscene, cams[v], trace_depth, pixel_offset=pixel_offset, outputs=("rgb", "paths"))
        g = d_rgb_fn(int(v), r["rgb"])
        a, b = api.render_backward(ctx, dscene, [cams[v]], trace_depth, r["paths"], g, pixel_offset=pixel_offset)
        gm += a
        gl += b
    return allreduce_grads(gm, gl)
