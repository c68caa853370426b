"""Thin torch.autograd.Function over eos_render / eos_render_backward (tests only).

Parameters are torch tensors: materials [K, 8] or [K, 10] (kd rgb, ks rgb, log shininess,
reflectivity[, transparency, refractive index]) and lights [L, 6] (position, colour).  Forward renders the views with the
plain renderer and keeps the path records; backward replays them with visibility frozen.
"""
import torch

from eos_b200 import api


class EosRender(torch.autograd.Function):
    @staticmethod
    def forward(fctx, mat_params, light_params, rctx, dscene, cams, trace_depth):
        mats = mat_params.detach().clone()
        mats[:, 6] = torch.exp(mats[:, 6])
        dscene.set_materials(mats.float().contiguous().cuda())
        dscene.set_lights(light_params.detach().float().contiguous().cuda())
        imgs, paths = [], []
        for c in cams:
            r = api.render(rctx, dscene, c, trace_depth, pixel_offset=0.5, outputs=("rgb", "paths"), device=True)
            imgs.append(r["rgb"])
            paths.append(r["paths"])
        fctx.save_for_backward(torch.cat(paths))
        fctx.rctx, fctx.dscene, fctx.cams, fctx.td = rctx, dscene, cams, trace_depth
        fctx.mat_shape = tuple(mat_params.shape)
        return torch.stack(imgs)

    @staticmethod
    def backward(fctx, grad_img):
        (paths,) = fctx.saved_tensors
        gm, gl = api.render_backward(fctx.rctx, fctx.dscene, fctx.cams, fctx.td, paths,
                                     grad_img.contiguous().float().reshape(-1, 3), pixel_offset=0.5)
        gmat = torch.zeros(fctx.mat_shape, device=gm.device, dtype=torch.float32)
        gmat[:, :7] = gm
        return gmat, gl, None, None, None, None
