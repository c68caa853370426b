"""GPU adjoint (eos_render_backward) against the FP64 CPU adjoint of the same renderer,
whose own correctness is checked against central differences in test_oracle.py."""
import numpy as np
import pytest

import oracle
from eos_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _rel_close(a, b, rel=1e-3):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.abs(b).max()
    return np.abs(a - b).max() <= rel * max(scale, 1e-12), (np.abs(a - b).max(), scale)


@pytest.mark.parametrize("td,transparent,spp", [(1, False, 1), (2, False, 1), (2, True, 1), (2, False, 2)])
def test_backward_matches_fp64_adjoint(ctx, td, transparent, spp):
    import torch
    sc = scenes.config4_scene()
    sc.materials[:, 7] = 0.3  # mirror bounces so reflected shading is differentiated too
    if transparent:  # every third object transparent: Fresnel-mixed secondary rays
        sc.materials[::3, 7] = 0.0
        sc.materials[::3, 8] = 1.0
        sc.materials[::3, 9] = 1.52
    dsc = api.DeviceScene(ctx, sc)
    cams = scenes.config4_cameras(2, 64)
    paths, rgb = [], []
    for c in cams:
        r = api.render(ctx, dsc, c, td, pixel_offset=0.5, spp=spp, jitter_seed=9, outputs=("rgb", "paths"),
                       device=True)
        paths.append(r["paths"])
        rgb.append(r["rgb"])
    paths = torch.cat(paths)
    rgb = torch.cat(rgb)
    rng = np.random.default_rng(4)
    target = torch.from_numpy(rng.uniform(0, 0.6, tuple(rgb.shape)).astype(np.float32)).cuda()
    g = 2.0 * (rgb - target)
    gm, gl = api.render_backward(ctx, dsc, cams, td, paths, g, pixel_offset=0.5, spp=spp, jitter_seed=9)
    torch.cuda.synchronize()
    mp = sc.materials.astype(np.float64).copy()
    mp[:, 6] = np.log(mp[:, 6])
    lp = sc.lights.astype(np.float64)
    orc = oracle.Oracle(sc)
    p = paths.cpu().numpy()
    rgb64, om, ol = orc.frozen_f64(cams, 64, 64, 0.5, td, p[:, :8], p[:, 8:].view(np.uint32), mp, lp,
                                   g=g.cpu().numpy().astype(np.float64), spp=spp, jitter_seed=9)
    # FP32 forward vs the FP64 re-render of the same frozen paths: colours up to ~4 with
    # shininess up to e^5, so pow() turns ~1e-7 direction rounding into ~1e-4 relative
    r32 = rgb.cpu().numpy()
    assert (np.abs(rgb64 - r32) / np.maximum(1.0, np.abs(rgb64))).max() < 1e-3
    gm = gm.cpu().numpy()
    gl = gl.cpu().numpy()
    for name, a, b in [("kd", gm[:, 0:3], om[:, 0:3]), ("ks", gm[:, 3:6], om[:, 3:6]),
                       ("log_shininess", gm[:, 6], om[:, 6]), ("light_colour", gl[:, 0:3], ol[:, 0:3]),
                       ("light_position", gl[:, 3:6], ol[:, 3:6])]:
        ok, info = _rel_close(a, b)
        assert ok, (name, info)


@pytest.mark.parametrize("spp", [1, 2])
def test_row_band_gradients_sum_to_the_frame(ctx, spp):
    """Split-frame differentiation: each band's forward records and loss gradient give that
    band's share, and the shares of three bands add up to the whole frame's gradients."""
    import torch
    sc = scenes.config4_scene()
    sc.materials[:, 7] = 0.3
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.config4_cameras(1, 64)[0]
    td = 2
    rng = np.random.default_rng(8)
    target = torch.from_numpy(rng.uniform(0, 0.6, (64 * 64, 3)).astype(np.float32)).cuda()
    r = api.render(ctx, dsc, cam, td, spp=spp, jitter_seed=4, outputs=("rgb", "paths"), device=True)
    g = 2.0 * (r["rgb"] - target)
    fm, fl = api.render_backward(ctx, dsc, [cam], td, r["paths"], g, spp=spp, jitter_seed=4)
    sm = torch.zeros_like(fm)
    sl = torch.zeros_like(fl)
    for r0, r1 in ((0, 20), (20, 41), (41, 64)):
        b = api.render(ctx, dsc, cam, td, spp=spp, jitter_seed=4, outputs=("rgb", "paths"), device=True,
                       rows=(r0, r1))
        assert torch.equal(b["rgb"], r["rgb"][r0 * 64:r1 * 64])
        gb = 2.0 * (b["rgb"] - target[r0 * 64:r1 * 64])
        bm, bl = api.render_backward(ctx, dsc, [cam], td, b["paths"], gb, spp=spp, jitter_seed=4, rows=(r0, r1))
        sm += bm
        sl += bl
    for a, b in ((sm, fm), (sl, fl)):  # float atomics sum in another order
        assert (a - b).abs().max() <= 1e-4 * b.abs().max()


def test_autograd_function_inverse_shading_reduces_loss(ctx):
    """Config-4 style inverse shading: a few gradient steps from perturbed parameters."""
    import torch
    from tests.autograd_fn import EosRender
    hidden = scenes.config4_scene()
    start = scenes.config4_scene(hidden=False)
    cams = scenes.config4_cameras(4, 64)
    dsc = api.DeviceScene(ctx, hidden)
    targets = torch.stack([api.render(ctx, dsc, c, 1, pixel_offset=0.5, outputs=("rgb",))["rgb"] for c in cams])
    m0 = torch.tensor(start.materials, dtype=torch.float32, device="cuda")
    m0[:, 6] = torch.log(m0[:, 6])
    mat = m0.clone().requires_grad_(True)
    lights = torch.tensor(start.lights, dtype=torch.float32, device="cuda").requires_grad_(True)
    opt = torch.optim.Adam([mat, lights], lr=0.02)
    losses = []
    for it in range(15):
        opt.zero_grad()
        img = EosRender.apply(mat, lights, ctx, dsc, cams, 1)
        loss = ((img - targets) ** 2).sum()
        loss.backward()
        with torch.no_grad():
            mat.grad[:, 7] = 0.0  # reflectivity is not a parameter
        opt.step()
        losses.append(float(loss))
    assert losses[-1] < 0.5 * losses[0], losses
