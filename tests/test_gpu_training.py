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
    bad = np.flatnonzero(~np.isfinite(history))
    assert bad.size == 0, ("non-finite step loss", int(bad[0]), history[max(0, bad[0] - 3):bad[0] + 2])
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


def test_training_loop_trajectory_matches_oracle():
    """The training-loop configuration at test size: a 6,000-point SH-degree-3
    teacher renders 16 targets (96x96, by the oracle); the perturbed student
    takes 12 multi-view graph-replayed steps of 8 views (lr_sh 2.5e-3, lr_verts
    1e-4, lr_dens 1e-2, lr_grads 1e-3, L2) on the GPU and in the oracle, and
    every step's per-view losses agree within 1e-3 relative."""
    import os

    from oracle import Oracle, OracleTrainer

    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene

    rng = np.random.default_rng(11)
    teacher = make_scene(gmm_cloud(6000, rng), rng, sh_degree=3)
    cams = orbit_cameras(16, seed=12, radius=(2.5, 4.0), resolutions=((96, 96),))
    orc = Oracle("f32")
    shv = orc.sh_values(teacher["sh_coeffs"])
    targets = [orc.forward_tiled(teacher, c, 12, sh=shv, sh_degree=3)["image"][..., :3].copy() for c in cams]

    prng = np.random.default_rng(13)
    student = dict(teacher)
    student["sh_coeffs"] = (teacher["sh_coeffs"] + prng.normal(0, 0.3, teacher["sh_coeffs"].shape)).astype(np.float32)
    student["densities"] = np.exp(np.log(teacher["densities"]) + prng.normal(0, 0.5, teacher["densities"].shape)
                                  ).astype(np.float32)
    student["vertices"] = (teacher["vertices"] + prng.normal(0, 0.01, teacher["vertices"].shape)).astype(np.float32)

    from rmesh_b200 import RMeshRenderer

    rs = RMeshRenderer(student["vertices"], student["indices"], student["base_colors"], student["densities"],
                       student["color_grads"], student["circumdata"], 96, 96, tile_size=12,
                       sh_coeffs=student["sh_coeffs"], sh_degree=3)
    tr = OracleTrainer(student, use_sh=True)
    lrs = (1e-4, 1e-2, 1e-3)
    threads = min(16, os.cpu_count() or 1)
    for step in range(12):
        sel = [(8 * step + j) % 16 for j in range(8)]
        vc = [cams[i] for i in sel]
        gts = [targets[i] for i in sel]
        lg = rs.train_step_views(vc, gts, *lrs, 1, mode="graph", lr_sh=2.5e-3)
        lo = tr.train_step_views(vc, gts, *lrs, 1, lr_sh=2.5e-3, threads=threads)
        rel = np.abs(lg - lo) / np.abs(lo)
        assert np.all(rel <= 1e-3), (step, lg, lo)
    assert rs.step == tr.step == 12
    rs.close()


def test_gradients_of_a_trained_student_match_oracle():
    """After 40 training steps (vertices moved, slivers and inverted tets from
    the N(0, 0.01) vertex perturbation of a dense mesh), a single-view adjoint
    on the trained parameters still matches the oracle's: images within 1e-4,
    gradients within 1e-3 relative L2 per group."""
    from oracle import Oracle

    from rmesh_b200 import RMeshRenderer
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene

    rng = np.random.default_rng(31)
    sc = make_scene(gmm_cloud(20000, rng), rng, sh_degree=3)
    prng = np.random.default_rng(32)
    sc["vertices"] = (sc["vertices"] + prng.normal(0, 0.01, sc["vertices"].shape)).astype(np.float32)
    cams = orbit_cameras(8, seed=33, radius=(2.5, 4.0), resolutions=((160, 160),))
    trng = np.random.default_rng(34)
    gts = [trng.uniform(0, 1, (160, 160, 3)).astype(np.float32) for _ in cams]
    r = RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 160, 160, tile_size=12, sh_coeffs=sc["sh_coeffs"], sh_degree=3)
    for _ in range(40):
        r.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1, mode="graph", lr_sh=2.5e-3)
    p = r.get_params()
    trained = dict(sc, vertices=p["vertices"], densities=p["densities"], color_grads=p["color_grads"],
                   sh_coeffs=p["sh_coeffs"])
    assert np.abs(p["vertices"] - sc["vertices"]).max() > 1e-3  # the vertices did move
    cam, gt = cams[0], gts[0]
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    dl = np.zeros((160, 160, 4), np.float32)
    dl[..., :3] = 2.0 * (img[..., :3] - gt) / (160 * 160)
    g = r.backward(dl)
    r.close()

    o = Oracle("f32")
    shv = o.sh_values(trained["sh_coeffs"])
    fo = o.forward_tiled(trained, cam, 12, sh=shv, sh_degree=3)
    assert np.abs(img - fo["image"]).max() <= 1e-4
    go = o.backward(trained, cam, dl, fo, 12, sh=shv, sh_degree=3)
    for k, ko in (("d_vertices", "d_vertices"), ("d_densities", "d_densities"), ("d_color_grads", "d_color_grads"),
                  ("d_sh_coeffs", "d_sh")):
        a, b = np.float64(g[k]), np.float64(go[ko])
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b), k
