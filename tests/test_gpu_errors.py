"""Device error paths, made to fire on ordinary scenes by the context's test limits
(eos_ctx_set_limits) -- no fault, trap or hang: each limited call returns its status, and
the same context renders the frame correctly right afterwards.

  queue_entries  -> EOS_ERR_QUEUE_OVERFLOW (6)
  work_budget    -> EOS_ERR_TIMEOUT (4), the persistent loops' iteration budget
  small_stack    -> EOS_ERR_STACK_OVERFLOW (5)
"""
import numpy as np
import pytest

from eos_b200 import api, scenes
from eos_b200._lib import EosError

pytestmark = pytest.mark.gpu

TIMEOUT, STACK, QUEUE = 4, 5, 6


@pytest.fixture(scope="module")
def big(ctx):
    """A 300k-triangle mixed scene: its 4-wide tree is deep enough for an 8-entry stack to
    overflow on shadow rays."""
    sc = scenes.mixed_scene(scenes.rng_for(4243), 300_000, "mixed300k")
    dsc = api.DeviceScene(ctx, sc)
    cam = scenes.look_at((0, 25, 60), (0, 0, 0), 60.0, 256, 192)
    ref = api.render(ctx, dsc, cam, 2, mode="wavefront", outputs=("rgb", "paths"), device=False)
    return dsc, cam, ref


class _Status(int):
    """The status of a limited call; its repr carries the library's error detail, so that a
    failed comparison shows which CUDA call or device error it was."""

    def __new__(cls, err):
        obj = super().__new__(cls, err.code)
        obj.detail = str(err)
        return obj

    def __repr__(self):
        return f"{int(self)} ({self.detail})"


def _limited(ctx, fn, **lim):
    ctx.set_limits(**lim)
    try:
        with pytest.raises(EosError) as e:
            fn()
        return _Status(e.value)
    finally:
        ctx.set_limits()


def _same(a, b):
    assert np.array_equal(a["paths"], b["paths"])
    assert np.array_equal(a["rgb"], b["rgb"])


@pytest.mark.parametrize("lim,code", [(dict(queue_entries=64), QUEUE), (dict(work_budget=1000), TIMEOUT),
                                      (dict(small_stack=True), STACK)])
def test_limit_gives_its_status_and_the_context_stays_usable(ctx, big, lim, code):
    dsc, cam, ref = big
    assert ref["stats"]["error_flags"] == 0
    # eos_render in wavefront mode
    got = _limited(ctx, lambda: api.render(ctx, dsc, cam, 2, mode="wavefront", outputs=("rgb", "paths"),
                                           device=False), **lim)
    assert got == code
    _same(api.render(ctx, dsc, cam, 2, mode="wavefront", outputs=("rgb", "paths"), device=False), ref)
    # eos_render_batch (graph-captured; the limits are part of the graph's key)
    jobs = [api.BatchJob(dsc, cam, 2, 0.5)]
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"))
    got = _limited(ctx, lambda: api.render_batch(ctx, jobs, outs), **lim)
    assert got == code
    outs = api.make_batch_outputs(jobs, ("rgb", "paths"))
    api.render_batch(ctx, jobs, outs)
    assert np.array_equal(outs[0]["paths"].cpu().numpy(), ref["paths"])
    assert np.array_equal(outs[0]["rgb"].cpu().numpy(), ref["rgb"])


@pytest.mark.parametrize("lim,code", [(dict(queue_entries=64), QUEUE), (dict(work_budget=1000), TIMEOUT),
                                      (dict(small_stack=True), STACK)])
def test_limits_on_a_pass_of_two_lanes(ctx, big, lim, code):
    """A view of more than 2^20 paths runs as two lanes (halves of its paths side by side):
    each limit still gives its status, and the same context then renders the plain
    renderer's image.  Before the limited call a batch of four jobs on a scene that is then
    destroyed fills the queues: a limited call reads none of those stale entries (a shadow
    queue entry names its job and hit, which would point into the destroyed scene)."""
    import torch
    dsc, _, _ = big
    cam = scenes.look_at((0, 25, 60), (0, 0, 0), 60.0, 1280, 960)
    ref = api.render(ctx, dsc, cam, 2, mode="plain", outputs=("rgb",), device=True)
    tmp = api.DeviceScene(ctx, scenes.small_random_scene(44, n_spheres=6, level=3, lights=8, refl=0.6))
    pre = [api.BatchJob(tmp, scenes.look_at((0.5 * k, 3.0, 9.0), (0, -0.5, 0), 55.0, 1280, 960), 2, 0.5)
           for k in range(4)]
    api.render_batch(ctx, pre, api.make_batch_outputs(pre, ("rgb",)))
    torch.cuda.synchronize()
    tmp.close()
    jobs = [api.BatchJob(dsc, cam, 2, 0.5)]
    outs = api.make_batch_outputs(jobs, ("rgb",))
    assert _limited(ctx, lambda: api.render_batch(ctx, jobs, outs), **lim) == code
    api.render_batch(ctx, jobs, outs)
    torch.cuda.synchronize()
    assert torch.equal(outs[0]["rgb"], ref["rgb"])


def test_work_budget_leaves_untraced_paths_marked(ctx, big):
    """Past the budget the queue entries stay untraced: their path records keep
    EOS_HIT_UNTRACED (-2) and the traced ones equal the unlimited render's."""
    dsc, cam, ref = big
    out = {}
    npx = cam.width * cam.height
    paths = np.zeros((npx, 16), np.int32)
    out["paths"] = paths
    ctx.set_limits(work_budget=4096)
    try:
        with pytest.raises(EosError) as e:
            api.render(ctx, dsc, cam, 2, mode="wavefront", outputs=(), out=out, device=False)
        assert e.value.code == TIMEOUT
    finally:
        ctx.set_limits()
    prim = paths[:, 0]
    traced = prim != -2
    assert 0 < traced.sum() < npx
    assert np.array_equal(prim[traced], ref["paths"][traced, 0])


def test_limits_reject_negative_values(ctx):
    with pytest.raises(EosError) as e:
        ctx.set_limits(queue_entries=-1)
    assert e.value.code == 1
    ctx.set_limits()
