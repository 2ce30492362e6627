"""Multi-process data parallelism on the CPU (gloo, world size 2).

The path's only exchange step is the sum of the ranks' gradients before Adam.
These tests run that exchange with the CPU oracle producing each rank's
gradients for its shard of views, and check the failure path: a rank that
leaves before the collective makes the survivor's all-reduce fail within the
process-group timeout instead of hanging.
"""
from __future__ import annotations

import datetime
import os
import socket
import sys

import numpy as np

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _scene_and_views():
    sys.path.insert(0, ROOT)
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import make_scene, uniform_cloud

    rng = np.random.default_rng(4)
    sc = make_scene(uniform_cloud(120, rng), rng)
    cams = orbit_cameras(4, seed=9, radius=(2.4, 3.0), resolutions=((32, 32), (40, 24)))
    trng = np.random.default_rng(5)
    gts = [trng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    return sc, cams, gts


def _grads_for(sc, cams, gts, views):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle

    o = Oracle("f32")
    tot = None
    for i in views:
        f = o.forward_tiled(sc, cams[i])
        _, dl = o.loss(f["image"], gts[i], 1)
        g = o.backward(sc, cams[i], dl, f)
        flat = np.concatenate([g[k] for k in ("d_vertices", "d_densities", "d_color_grads", "d_base_colors")])
        tot = flat if tot is None else tot + flat
    return tot


def _worker(rank, world, port, outdir, fail_rank):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from rmesh_b200.dp import allreduce_sum_, shard_views

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=15))
    sc, cams, gts = _scene_and_views()
    local = _grads_for(sc, cams, gts, shard_views(len(cams), world, rank))
    if rank == fail_rank:
        os._exit(3)  # leaves between steps, before the collective
    t = torch.from_numpy(local.astype(np.float32))
    try:
        allreduce_sum_(t)
        np.save(os.path.join(outdir, f"grad_{rank}.npy"), t.numpy())
    except Exception as e:  # the survivor learns of the departure from the collective
        with open(os.path.join(outdir, f"error_{rank}.txt"), "w") as f:
            f.write(type(e).__name__ + ": " + str(e)[:200])
    dist.destroy_process_group() if fail_rank < 0 else None


def _run(world, outdir, fail_rank=-1, timeout=120):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, outdir, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
        if p.is_alive():
            p.kill()
            raise AssertionError("worker did not finish")
    return [p.exitcode for p in procs]


def test_gradient_allreduce_equals_serial_sum(tmp_path):
    codes = _run(2, str(tmp_path))
    assert codes == [0, 0]
    g0 = np.load(tmp_path / "grad_0.npy")
    g1 = np.load(tmp_path / "grad_1.npy")
    np.testing.assert_array_equal(g0, g1)  # every rank holds the same summed gradient
    sc, cams, gts = _scene_and_views()
    serial = _grads_for(sc, cams, gts, range(len(cams)))
    err = np.linalg.norm(g0.astype(np.float64) - serial) / np.linalg.norm(serial)
    assert err < 1e-5, err


def test_departed_rank_is_detected(tmp_path):
    codes = _run(2, str(tmp_path), fail_rank=1)
    assert codes[1] == 3
    errs = list(tmp_path.glob("error_0.txt"))
    assert errs, "rank 0 did not observe the failure"
    assert not (tmp_path / "grad_0.npy").exists()
