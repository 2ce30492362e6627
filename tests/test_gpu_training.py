"""Teacher-student training (the training-loop configuration, reduced to test
size; needs a B200): a teacher mesh renders targets, a student with the same
topology and perturbed parameters (SH + N(0, 0.3), log-density + N(0, 0.5),
vertices + N(0, 0.01)) is fitted with multi-view Adam steps (lr_sh 2.5e-3,
lr_verts 1e-4, lr_dens 1e-2, lr_grads 1e-3, L2), and its loss must fall and
its image of a held-out view move toward the teacher's."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_student_converges_toward_teacher():
    import torch

    from rmesh_b200 import RMeshRenderer
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene

    rng = np.random.default_rng(5)
    teacher = make_scene(gmm_cloud(6000, rng), rng, sh_degree=3)
    cams = orbit_cameras(16, seed=6, radius=(2.5, 3.5), resolutions=((192, 192),))
    kw = dict(tile_size=12, sh_coeffs=teacher["sh_coeffs"], sh_degree=3)
    rt = RMeshRenderer(teacher["vertices"], teacher["indices"], teacher["base_colors"], teacher["densities"],
                       teacher["color_grads"], teacher["circumdata"], 192, 192, **kw)
    targets = [rt.forward_tiled(c.cam_pos, c.vp, c.c2w_intrinsics)[..., :3].copy() for c in cams]
    rt.close()

    prng = np.random.default_rng(7)
    student = dict(teacher)
    student["sh_coeffs"] = (teacher["sh_coeffs"] + prng.normal(0, 0.3, teacher["sh_coeffs"].shape)).astype(np.float32)
    student["densities"] = np.exp(np.log(teacher["densities"]) + prng.normal(0, 0.5, teacher["densities"].shape)
                                  ).astype(np.float32)
    student["vertices"] = (teacher["vertices"] + prng.normal(0, 0.01, teacher["vertices"].shape)).astype(np.float32)
    rs = RMeshRenderer(student["vertices"], student["indices"], student["base_colors"], student["densities"],
                       student["color_grads"], student["circumdata"], 192, 192, tile_size=12,
                       sh_coeffs=student["sh_coeffs"], sh_degree=3)
    gts = torch.from_numpy(np.stack(targets)).cuda()
    history = []
    for step in range(150):
        sel = [(4 * step + j) % 16 for j in range(4)]  # 4 views per step, cycling through the 16
        gt = gts[sel].reshape(-1).contiguous()
        losses = rs.train_step_views([cams[i] for i in sel], gt, 1e-4, 1e-2, 1e-3, 1, mode="graph", lr_sh=2.5e-3)
        history.append(float(np.mean(losses)))
    first, last = np.mean(history[:4]), np.mean(history[-8:])
    assert np.all(np.isfinite(history))
    assert last < 0.5 * first, (first, last)
    assert rs.step == 150
    # a held-out view: the student's image moved toward the teacher's
    hold = orbit_cameras(1, seed=99, radius=(3.0, 3.0), resolutions=((192, 192),))[0]
    rt = RMeshRenderer(teacher["vertices"], teacher["indices"], teacher["base_colors"], teacher["densities"],
                       teacher["color_grads"], teacher["circumdata"], 192, 192, **kw)
    want = rt.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics)
    r0 = RMeshRenderer(student["vertices"], student["indices"], student["base_colors"], student["densities"],
                       student["color_grads"], student["circumdata"], 192, 192, tile_size=12,
                       sh_coeffs=student["sh_coeffs"], sh_degree=3)
    before = np.abs(r0.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics) - want).mean()
    after = np.abs(rs.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics) - want).mean()
    assert after < 0.95 * before, (before, after)
