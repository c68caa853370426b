"""Comparison helpers shared by the parity tests."""
from __future__ import annotations

import numpy as np

import oracle

RGB_TOL = 1e-4  # max-abs FP32 colour tolerance before 8-bit quantisation


def primary_rays(cam, pixel_offset=0.0, pixels=None):
    """Primary rays in the reference's float order (src/RayTracer.cpp:119-145)."""
    W, H = cam.width, cam.height
    p = np.arange(W * H) if pixels is None else np.asarray(pixels)
    x = (p % W).astype(np.float32)
    y = (p // W).astype(np.float32)
    nw, nh = np.float32(W / 2.0), np.float32(H / 2.0)
    inw, inh = np.float32(1.0) / nw, np.float32(1.0) / nh
    off = np.float32(pixel_offset)
    bb = ((y + off) - nh) * inh
    aa = ((x + off) - nw) * inw
    d = (aa[:, None] * cam.right[None, :] + bb[:, None] * cam.up[None, :]) + cam.view[None, :]
    dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    s = np.float32(1.0) / np.sqrt(dd)
    d = d * s[:, None]
    o = np.broadcast_to(cam.position, d.shape)
    return np.concatenate([o, d], 1).astype(np.float32)


def path_mismatch(hits_a, sh_a, hits_b, sh_b, nb):
    """Boolean per path: hit ids or shadow masks differ within the first nb bounces."""
    ha = np.asarray(hits_a)[:, :nb]
    hb = np.asarray(hits_b)[:, :nb]
    sa = np.asarray(sh_a)[:, :nb].astype(np.uint32)
    sb = np.asarray(sh_b)[:, :nb].astype(np.uint32)
    return (ha != hb).any(1) | (sa != sb).any(1)


def classify(mismatch, flags):
    """Splits mismatching paths into the oracle's flagged classes and unexplained ones."""
    flags = np.asarray(flags)
    out = {
        "paths": int(mismatch.size),
        "mismatch": int(mismatch.sum()),
        "tie_2ulp": int((mismatch & ((flags & oracle.FLAG_TIE) != 0)).sum()),
        "axis_parallel": int((mismatch & ((flags & oracle.FLAG_AXIS_PARALLEL) != 0)).sum()),
        "near_origin": int((mismatch & ((flags & oracle.FLAG_NEAR_ORIGIN) != 0)).sum()),
        "unexplained": int((mismatch & (flags == 0)).sum()),
    }
    # the classes beyond the 2-ulp rule: flagged paths that are not also near ties
    no_tie = mismatch & ((flags & oracle.FLAG_TIE) == 0)
    out["axis_parallel_not_tie"] = int((no_tie & ((flags & oracle.FLAG_AXIS_PARALLEL) != 0)).sum())
    out["near_origin_not_tie"] = int((no_tie & ((flags & oracle.FLAG_NEAR_ORIGIN) != 0)).sum())
    return out
