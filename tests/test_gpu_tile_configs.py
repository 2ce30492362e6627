"""Tile configurations (tile size x threads per tile, per resolution) and the
grid autotuner on the CUDA path vs the CPU oracle (needs a B200).

Every configuration must give the oracle's results at that tile size: bit-exact
binning, images within 1e-4, gradients within 1e-3 relative L2; a multi-view
step whose resolutions run different configurations (one persistent launch per
configuration) must give each view the loss and gradients it has alone.
Design input for the grid: crates/rmesh-backward/examples/tile_size_sweep.rs:1-60.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import c1_camera, make_renderer, rel_l2

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-4
GRAD_TOL = 1e-3
CONFIGS = [(8, 64), (8, 128), (12, 160), (12, 320), (16, 256), (16, 512)]


@pytest.mark.parametrize("ts,threads", CONFIGS)
def test_every_configuration_matches_oracle(c1_scene, oracle32, ts, threads):
    cam = c1_camera(200, 136)
    r = make_renderer(c1_scene, cam, tile_size=ts)
    r.set_tile_config(ts, threads)
    assert r.tile_config() == (ts, threads)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(c1_scene, cam, tile_size=ts)
    np.testing.assert_array_equal(r.debug_tiles_touched(), np.where(ref["visible"] > 0, ref["tiles_touched"], 0))
    tiles, tets = r.debug_pairs()
    np.testing.assert_array_equal(tiles, ref["key_hi"])
    np.testing.assert_array_equal(tets, ref["vals"])
    assert np.abs(img - ref["image"]).max() <= IMG_TOL
    gt = np.random.default_rng(ts).uniform(0, 1, (cam.height, cam.width, 3)).astype(np.float32)
    _, dl = oracle32.loss(ref["image"], gt, 1)
    g = r.backward(dl)
    go = oracle32.backward(c1_scene, cam, dl, ref, tile_size=ts, threads=oracle32.max_threads)
    for k in ("d_vertices", "d_densities", "d_color_grads", "d_base_colors"):
        assert rel_l2(g[k], go[k]) <= GRAD_TOL, k
    r.close()


def _mixed_views():
    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(5, seed=31, radius=(2.5, 3.5), resolutions=((96, 96), (160, 120), (64, 64)))
    rng = np.random.default_rng(9)
    gts = [rng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    return cams, gts


def _oracle_step(oracle, scene, cams, gts, plan):
    """Per-view losses and summed gradients of the oracle, each view at the
    tile size its configuration uses."""
    losses, total = [], None
    for c, gt in zip(cams, gts):
        ts = plan.get((c.width, c.height), (12, 0))[0]
        f = oracle.forward_tiled(scene, c, tile_size=ts)
        loss, dl = oracle.loss(f["image"], gt, 1)
        g = oracle.backward(scene, c, dl, f, tile_size=ts, threads=oracle.max_threads)
        losses.append(loss)
        total = g if total is None else {k: total[k] + g[k] for k in total}
    return np.array(losses), total


@pytest.mark.parametrize("mode", ["plain", "batched", "graph"])
def test_per_resolution_configurations_in_one_step(c1_scene, oracle32, mode):
    cams, gts = _mixed_views()
    plan = {(96, 96): (8, 128), (160, 120): (16, 256), (64, 64): (12, 320)}
    r = make_renderer(c1_scene, cams[0])
    for (w, h), (ts, th) in plan.items():
        r.set_resolution_tile_config(w, h, ts, th)
        assert r.tile_config(w, h) == (ts, th)
    want_l, want_g = _oracle_step(oracle32, c1_scene, cams, gts, plan)
    for _ in range(2):  # graph mode: capture, then replay
        losses = r.accumulate_views(cams, gts, 1, mode=mode)
        np.testing.assert_allclose(losses, want_l, rtol=1e-4)
    slots = r.grad_slots().cpu().numpy()
    m = c1_scene["densities"].size
    s = slots[:20 * m].reshape(m, 20).astype(np.float64)
    np.testing.assert_allclose(rel_l2(s[:, 0], want_g["d_densities"]), 0.0, atol=GRAD_TOL)
    np.testing.assert_allclose(rel_l2(s[:, 4:7].ravel(), want_g["d_color_grads"]), 0.0, atol=GRAD_TOL)
    # removing an override returns that resolution to the default
    r.set_resolution_tile_config(96, 96, 0)
    assert r.tile_config(96, 96) == r.tile_config()
    r.close()


def test_grid_autotune(c1_scene):
    cams, gts = _mixed_views()
    r = make_renderer(c1_scene, cams[0])
    before = r.get_params()
    out = r.autotune(cams, gts)
    grid = out["grid"]
    uniform = [e for e in grid if e["views"] == "all"]
    assert [(e["tile_size"], e["threads"]) for e in uniform] == CONFIGS
    assert all(e["ms"] > 0 for e in grid)
    per_res = [e for e in grid if "x" in e["views"]]
    assert len(per_res) == 3 * len(CONFIGS)
    best = min(uniform, key=lambda e: e["ms"])
    assert out["chosen"]["default"] == (best["tile_size"], best["threads"])
    after = r.get_params()
    for k in before:
        np.testing.assert_array_equal(before[k], after[k])
    losses = r.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1, mode="graph")
    assert np.all(np.isfinite(losses)) and r.step == 1
    r.close()
