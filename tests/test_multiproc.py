"""Multi-process (gloo, world size 2, CPU) tests of the view sharding and the gradient
all-reduce: the sharded sum over ranks equals the single-process adjoint."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle
from eos_b200 import parallel, scenes


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _setup():
    sc = scenes.small_random_scene(71, n_spheres=4, level=2, lights=2, refl=0.4)
    cams = [scenes.look_at((6 * np.cos(a), 3.0, 6 * np.sin(a)), (0, -0.5, 0), 55.0, 16, 12)
            for a in np.linspace(0, 2 * np.pi, 5, endpoint=False)]
    return sc, cams


def _grads_for_views(sc, cams, views):
    orc = oracle.Oracle(sc)
    mp_ = sc.materials.astype(np.float64).copy()
    mp_[:, 6] = np.log(mp_[:, 6])
    lp = sc.lights.astype(np.float64)
    gm = np.zeros((sc.n_objects, 7))
    gl = np.zeros((sc.n_lights, 6))
    for v in views:
        r = orc.render(cams[v], 1, pixel_offset=0.5)
        rng = np.random.default_rng(100 + v)
        g = rng.normal(size=(cams[v].width * cams[v].height, 3))
        _, a, b = orc.frozen_f64([cams[v]], cams[v].width, cams[v].height, 0.5, 1, r["hits"], r["shadows"], mp_, lp,
                                 g=g, nthreads=1)
        gm += a
        gl += b
    return gm, gl


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sc, cams = _setup()
    mine = parallel.shard_indices(len(cams), rank, world)
    gm, gl = _grads_for_views(sc, cams, mine)
    gm, gl = parallel.allreduce_grads(gm, gl)
    out[rank] = (gm, gl, list(mine))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_adjoint_allreduce_equals_single_process():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    sc, cams = _setup()
    gm_ref, gl_ref = _grads_for_views(sc, cams, range(len(cams)))
    assert sorted(res[0][2] + res[1][2]) == list(range(len(cams)))
    for r in range(world):
        np.testing.assert_allclose(res[r][0], gm_ref, rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(res[r][1], gl_ref, rtol=1e-9, atol=1e-12)


def test_shard_round_robin_covers_everything_once():
    items = list(range(11))
    parts = [parallel.shard(items, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == items
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def _band_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sc, cams = _setup()
    cam = cams[1]
    r0, r1 = parallel.band(cam.height, rank, world)
    # the oracle renders this rank's rows (its pixel list), as a GPU rank renders its band
    pix = np.arange(r0 * cam.width, r1 * cam.width)
    rgb = oracle.Oracle(sc).render(cam, 1, pixel_offset=0.5, pixels=pix, nthreads=1)["rgb"]
    full = parallel.gather_bands(rgb.reshape(r1 - r0, cam.width, 3), cam.height)
    out[rank] = (r0, r1, full)
    dist.barrier()
    dist.destroy_process_group()


def test_split_frame_bands_gather_to_the_whole_frame():
    world = 3  # 12 rows over 3 ranks: 4 + 4 + 4; and a remainder case below
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_band_worker, args=(world, port, out), nprocs=world, start_method="spawn")
    sc, cams = _setup()
    whole = oracle.Oracle(sc).render(cams[1], 1, pixel_offset=0.5, nthreads=1)["rgb"].reshape(12, 16, 3)
    for r in range(world):
        r0, r1, full = out[r]
        assert (r0, r1) == parallel.band(12, r, world)
        assert np.array_equal(full, whole)
    assert [parallel.band(10, r, 3) for r in range(3)] == [(0, 3), (3, 6), (6, 10)]
