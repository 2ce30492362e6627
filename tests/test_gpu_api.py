"""The rest of RMeshRenderer's surface on the GPU (lib.rs:2641-2705 and the
additions of this binding): update_params / get_params round trips and their
effect on rendering, SH coefficient updates and sh_grad_into, set_tile_size
after construction, the device-tensor backward_into, the stage profiler,
checkpoint / resume through state_dict, and run-to-run determinism of the
forward and the binning."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import c1_camera, make_renderer, rel_l2

pytestmark = pytest.mark.gpu


def _perturbed(scene, seed):
    rng = np.random.default_rng(seed)
    return {
        "vertices": (scene["vertices"] + rng.normal(0, 0.004, scene["vertices"].shape)).astype(np.float32),
        "base_colors": rng.uniform(0.1, 0.9, scene["base_colors"].shape).astype(np.float32),
        "densities": (scene["densities"] * rng.uniform(0.5, 1.5, scene["densities"].shape)).astype(np.float32),
        "color_grads": rng.normal(0, 0.1, scene["color_grads"].shape).astype(np.float32),
    }


def test_update_params_roundtrip_and_render(c1_scene):
    """update_params writes the four groups (None leaves a group as it is),
    get_params reads them back exactly, and the image equals that of a
    renderer constructed with the same parameters bit for bit."""
    cam = c1_camera(96, 96)
    new = _perturbed(c1_scene, 11)
    r = make_renderer(c1_scene, cam)
    r.update_params(new["vertices"], new["base_colors"], new["densities"], new["color_grads"])
    p = r.get_params()
    for k in new:
        np.testing.assert_array_equal(p[k], new[k], err_msg=k)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    r2 = make_renderer(dict(c1_scene, **new), cam)  # circumdata is a fixed input in both
    np.testing.assert_array_equal(img, r2.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics))
    r.update_params(None, None, c1_scene["densities"], None)
    p2 = r.get_params()
    np.testing.assert_array_equal(p2["densities"], c1_scene["densities"])
    np.testing.assert_array_equal(p2["vertices"], new["vertices"])
    with pytest.raises(ValueError):
        r.update_params(new["vertices"][:-3], None, None, None)
    r.close()
    r2.close()


def test_update_sh_and_sh_grad_into(c2_scene):
    """SH coefficients: update_params(sh_coeffs=...) then get_params, the image
    of the updated renderer equals a freshly built one, and sh_grad_into
    returns the backward's coefficient gradient."""
    cam = c1_camera(96, 80)
    sh = (c2_scene["sh_coeffs"] + 0.1).astype(np.float32)
    r = make_renderer(c2_scene, cam, sh=True)
    r.update_params(None, None, None, None, sh_coeffs=sh)
    np.testing.assert_array_equal(r.get_params()["sh_coeffs"], sh)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    r2 = make_renderer(dict(c2_scene, sh_coeffs=sh), cam, sh=True)
    np.testing.assert_array_equal(img, r2.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics))
    dl = np.random.default_rng(12).normal(0, 1e-4, (80, 96, 4)).astype(np.float32)
    g = r.backward(dl)
    out = np.empty_like(g["d_sh_coeffs"])
    r.sh_grad_into(out)
    np.testing.assert_array_equal(out, g["d_sh_coeffs"])
    assert np.abs(out).max() > 0
    r.close()
    r2.close()


def test_set_tile_size_after_construction(c1_scene):
    """set_tile_size(8) on a tile-12 renderer renders exactly as a renderer
    built with tile 8, and the info reports the new size."""
    cam = c1_camera(100, 76)
    r = make_renderer(c1_scene, cam, tile_size=12)
    r.set_tile_size(8)
    assert r.info().tile_size == 8
    r8 = make_renderer(c1_scene, cam, tile_size=8)
    np.testing.assert_array_equal(r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics),
                                  r8.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics))
    with pytest.raises(Exception):
        r.set_tile_size(10)
    r.close()
    r8.close()


def test_backward_into_device_tensors(c1_scene):
    """backward_into writes the four gradient groups into caller-owned CUDA
    tensors; they equal backward's arrays (up to float-atomic order)."""
    import torch

    cam = c1_camera(96, 96)
    r = make_renderer(c1_scene, cam)
    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    dl = np.random.default_rng(13).normal(0, 1e-4, (96, 96, 4)).astype(np.float32)
    g = r.backward(dl)
    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    outs = {k: torch.zeros(v.size, dtype=torch.float32, device="cuda") for k, v in g.items()}
    r.backward_into(torch.from_numpy(dl).cuda(), outs["d_vertices"], outs["d_densities"], outs["d_base_colors"],
                    outs["d_color_grads"])
    torch.cuda.synchronize()
    for k in ("d_vertices", "d_densities", "d_base_colors", "d_color_grads"):
        assert rel_l2(outs[k].cpu().numpy(), g[k]) <= 1e-6, k
    r.close()


def test_stage_profiler(c1_scene):
    """With profiling on, a batched step reports positive CUDA-event times for
    its stages and the kernels it launched; stage_times resets the counters."""
    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(2, seed=14, radius=(2.6, 3.4), resolutions=((96, 96),))
    gts = [np.random.default_rng(15).uniform(0, 1, (96, 96, 3)).astype(np.float32) for _ in cams]
    r = make_renderer(c1_scene, cams[0])
    r.stage_times()
    r.set_profiling(True)
    r.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1, mode="batched")
    ms, n, total = r.stage_times()
    r.set_profiling(False)
    for k in ("project", "emit", "pair_sort", "composite", "adam"):
        assert ms[k] > 0 and n[k] >= 1, k
    assert total >= sum(n.values())
    ms2, n2, total2 = r.stage_times()
    assert total2 == 0 and all(v == 0 for v in n2.values())
    r.close()


def test_checkpoint_resume_continues_the_run(c2_scene):
    """state_dict after three graph-mode steps; the original renderer takes
    three more.  A fresh renderer restored with load_state_dict takes the
    same three steps: per-view losses and parameters follow the original's
    (to float-atomic order).  Restoring the parameters alone (Adam moments and
    step at zero) lands measurably elsewhere."""
    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(3, seed=61, radius=(2.6, 3.4), resolutions=((96, 96), (80, 64)))
    rng = np.random.default_rng(62)
    gts = [rng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    lr = dict(lr_verts=1e-4, lr_dens=1e-2, lr_grads=1e-3, loss_type=1, mode="graph", lr_sh=2.5e-3)
    r = make_renderer(c2_scene, cams[0], sh=True)
    for _ in range(3):
        r.train_step_views(cams, gts, **lr)
    st = r.state_dict()
    assert st["step"] == 3 and st["adam"].size > 0 and np.abs(st["adam"]).max() > 0
    la = [r.train_step_views(cams, gts, **lr) for _ in range(3)]
    pa = r.get_params()

    r2 = make_renderer(c2_scene, cams[0], sh=True)
    r2.load_state_dict(st)
    assert r2.step == 3
    lb = [r2.train_step_views(cams, gts, **lr) for _ in range(3)]
    pb = r2.get_params()
    for a, b in zip(la, lb):
        np.testing.assert_allclose(a, b, rtol=1e-5)

    r3 = make_renderer(c2_scene, cams[0], sh=True)
    p0 = st["params"]
    r3.update_params(p0["vertices"], p0["base_colors"], p0["densities"], p0["color_grads"], sh_coeffs=p0["sh_coeffs"])
    for _ in range(3):
        r3.train_step_views(cams, gts, **lr)
    pc = r3.get_params()
    for k in ("vertices", "densities", "color_grads", "sh_coeffs"):
        resumed, params_only = rel_l2(pb[k], pa[k]), rel_l2(pc[k], pa[k])
        assert resumed <= 1e-4, (k, resumed)
        assert params_only > 10 * max(resumed, 1e-9), (k, resumed, params_only)
    with pytest.raises(ValueError):
        r2.load_state_dict(dict(st, adam=st["adam"][:-1]))
    for x in (r, r2, r3):
        x.close()


def test_forward_and_binning_are_deterministic(c1_scene):
    """Two renderers over the same scene, and two calls on one renderer, give
    bit-identical images, tile counts and sorted (tile, tet) lists: the
    compaction is a chained scan and every sort is stable."""
    cam = c1_camera(128, 96)
    r1 = make_renderer(c1_scene, cam)
    r2 = make_renderer(c1_scene, cam)
    outs = []
    for r in (r1, r1, r2):
        img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
        tiles, tets = r.debug_pairs()
        outs.append((img, r.debug_tiles_touched(), tiles, tets))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            np.testing.assert_array_equal(a, b)
    r1.close()
    r2.close()


def test_out_of_range_index_rejected_on_the_device(c1_scene):
    """Indices passed as a CUDA tensor with one index equal to the vertex
    count: rmesh_create's range check (it reads only the index array) rejects
    them before any kernel gathers through them, and the device keeps
    rendering correctly."""
    import torch

    from rmesh_b200 import RMeshError, RMeshRenderer

    sc = c1_scene
    idx = torch.from_numpy(sc["indices"].astype(np.int32)).cuda()
    idx[7] = sc["vertices"].size // 3
    with pytest.raises(RMeshError):
        RMeshRenderer(sc["vertices"], idx, sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 64, 64)
    cam = c1_camera(64, 64)
    r = make_renderer(sc, cam)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    assert np.isfinite(img).all() and img[..., 3].max() > 0
    r.close()
