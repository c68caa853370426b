"""Multi-GPU plumbing: one process per GPU, views sharded across ranks.

Rendering shards with no data-path collective: views are independent, every rank
renders its own (the reference replicates the scene per GPU and splits frames by rows,
src/MultiDeviceRenderer.cu:59-81,119-161).  The adjoint has one real exchange step: the
parameter-gradient vector (per-object kd/ks/log-shininess, per-light colour/position) is
summed over ranks with one all-reduce.
"""
from __future__ import annotations

import numpy as np


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (balances uneven view sizes)."""
    return list(items)[rank::world]


def shard_indices(n: int, rank: int, world: int) -> np.ndarray:
    return np.arange(rank, n, world)


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
    K = dscene.scene.n_objects
    NL = max(1, dscene.scene.n_lights)
    gm = torch.zeros((K, 7), device="cuda")
    gl = torch.zeros((NL, 6), device="cuda")
    for v in mine:
        r = api.render(ctx, dscene, cams[v], trace_depth, pixel_offset=pixel_offset, outputs=("rgb", "paths"))
        g = d_rgb_fn(int(v), r["rgb"])
        a, b = api.render_backward(ctx, dscene, [cams[v]], trace_depth, r["paths"], g, pixel_offset=pixel_offset)
        gm += a
        gl += b
    return allreduce_grads(gm, gl)
