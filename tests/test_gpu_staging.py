"""Targets uploaded through ``TargetStager`` (pinned host memory, copy stream,
two device buffers) train as the same targets already on the device:
per-step losses and final parameters agree to rounding over graph-replayed
steps that alternate the two buffers (one cached CUDA graph per buffer), and
a stager refuses to refill a buffer whose targets no step has used."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene_and_views():
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene

    rng = np.random.default_rng(21)
    scene = make_scene(gmm_cloud(3000, rng), rng, sh_degree=2)
    cams = orbit_cameras(4, seed=22, radius=(2.5, 3.5), resolutions=((128, 96), (160, 160)))
    return scene, cams


def _renderer(scene):
    from rmesh_b200 import RMeshRenderer

    return RMeshRenderer(scene["vertices"], scene["indices"], scene["base_colors"], scene["densities"],
                         scene["color_grads"], scene["circumdata"], 128, 96, tile_size=12,
                         sh_coeffs=scene["sh_coeffs"], sh_degree=2)


def test_staged_targets_train_like_device_targets():
    import torch

    from rmesh_b200 import TargetStager

    scene, cams = _scene_and_views()
    n = sum(3 * c.width * c.height for c in cams)
    rng = np.random.default_rng(23)
    # a different target set per step, so a step reading the wrong buffer shows
    targets = [rng.random(n, dtype=np.float32) for _ in range(6)]
    lr = dict(lr_verts=1e-4, lr_dens=1e-2, lr_grads=1e-3, loss_type=1, mode="graph", lr_sh=2.5e-3)

    ra = _renderer(scene)
    stager = TargetStager(ra, n)
    host = [torch.from_numpy(t).pin_memory() for t in targets]
    la = []
    nxt = stager.put(host[0])
    for i in range(len(host)):
        cur = nxt
        if i + 1 < len(host):
            nxt = stager.put(host[i + 1])
        la.append(ra.train_step_views(cams, cur, **lr))
    with pytest.raises(ValueError):
        ra.train_step_views(cams, cur, **lr)  # a handle is used once
    pa = ra.get_params()

    rb = _renderer(scene)
    lb = [rb.train_step_views(cams, torch.from_numpy(t).cuda(), **lr) for t in targets]
    pb = rb.get_params()

    # losses and gradients are summed with float atomics, so two runs agree to
    # rounding, not bitwise; a step that read another step's (independent,
    # uniform) targets would move its loss by far more than 1e-5
    for a, b in zip(la, lb):
        np.testing.assert_allclose(a, b, rtol=1e-5)
    # an Adam update moves a parameter by at most about lr per step
    bound = {"vertices": 1e-4, "densities": 1e-2, "color_grads": 1e-3, "base_colors": 0.0, "sh_coeffs": 2.5e-3}
    for k in pa:
        np.testing.assert_allclose(pa[k], pb[k], rtol=0, atol=2 * bound[k] * len(targets) + 1e-6, err_msg=k)
    assert ra.step == rb.step == len(targets)

    # both buffers filled and unused: a third put must refuse
    s2 = TargetStager(ra, n)
    s2.put(host[0])
    s2.put(host[1])
    with pytest.raises(ValueError):
        s2.put(host[2])
    torch.cuda.synchronize()
    ra.close()
    rb.close()


def test_graph_cache_evicts_and_recaptures(c1_scene):
    """Ten device target buffers cycled through graph-mode steps: more
    signatures than the cache keeps (eight), so graphs are evicted and captured
    again; every step's losses and the final parameters equal batched mode's."""
    import torch

    from conftest import make_renderer, rel_l2

    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(2, seed=41, radius=(2.6, 3.4), resolutions=((96, 80), (64, 64)))
    n = sum(3 * c.width * c.height for c in cams)
    rng = np.random.default_rng(42)
    bufs = [torch.from_numpy(rng.uniform(0, 1, n).astype(np.float32)).cuda() for _ in range(10)]
    lr = dict(lr_verts=1e-4, lr_dens=1e-2, lr_grads=1e-3, loss_type=1)
    rg = make_renderer(c1_scene, cams[0])
    rb = make_renderer(c1_scene, cams[0])
    for i in range(23):
        gt = bufs[(3 * i) % 10]
        lg = rg.train_step_views(cams, gt, mode="graph", **lr)
        lb = rb.train_step_views(cams, gt, mode="batched", **lr)
        np.testing.assert_allclose(lg, lb, rtol=1e-4, err_msg=str(i))
    pg, pb = rg.get_params(), rb.get_params()
    for k in pg:
        assert rel_l2(pg[k], pb[k]) <= 1e-3, k
    rg.close()
    rb.close()
