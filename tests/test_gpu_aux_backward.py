"""Gradient of the custom aux channels on the CUDA path vs the CPU oracle (needs a B200).

The forward composites each custom channel as aux += T * alpha * a[tet]
(rasterize_compute.wgsl:458-462).  ``backward(dl_d_image, dl_d_aux)`` takes the
loss gradient of those channels, as the reference's ``dl_d_aux`` argument
(crates/rmesh-python/src/lib.rs:2043-2090), returns ``d_aux_data`` and adds the
channels' optical-depth terms to every other group.  The oracle's adjoint of
the same sum is pinned by float64 central differences
(tests/test_oracle.py::test_aux_channel_fd_gradients).  Bar: relative L2
<= 1e-3 per group.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import c1_camera, rel_l2, two_tet_scene

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-3
GROUPS = ("d_vertices", "d_densities", "d_color_grads", "d_base_colors", "d_aux_data")


def _renderer(sc, cam, aux_dim, ad):
    from rmesh_b200 import RMeshRenderer

    r = RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], cam.width, cam.height, aux_dim=aux_dim)
    r.set_aux_data(ad)
    return r


@pytest.mark.parametrize("aux_dim,res", [(3, (512, 512)), (1, (200, 120)), (8, (256, 256))])
def test_aux_backward_matches_oracle(c1_scene, oracle32, aux_dim, res):
    sc = c1_scene
    cam = c1_camera(*res)
    m = sc["densities"].size
    rng = np.random.default_rng(aux_dim)
    ad = rng.uniform(-1, 1, aux_dim * m).astype(np.float32)
    r = _renderer(sc, cam, aux_dim, ad)
    img, aux = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics, render_aux=True)
    ref = oracle32.forward_tiled(sc, cam, aux=True, aux_data=ad)
    assert np.abs(aux[..., 8:] - ref["aux"][..., 8:]).max() <= 1e-4
    gt = rng.uniform(0, 1, (cam.height, cam.width, 3)).astype(np.float32)
    _, dl = oracle32.loss(ref["image"], gt, 1)
    dl_aux = rng.normal(0, 1.0 / (cam.width * cam.height), (cam.height, cam.width, aux_dim)).astype(np.float32)
    g = r.backward(dl, dl_aux)
    go = oracle32.backward(sc, cam, dl, ref, threads=oracle32.max_threads, aux_data=ad, dl_aux=dl_aux)
    for k in GROUPS:
        e = rel_l2(g[k], go[k])
        assert e <= GRAD_TOL, (k, e)
    # the aux terms matter: without them the densities' gradient differs
    g0 = oracle32.backward(sc, cam, dl, ref, threads=oracle32.max_threads)
    assert rel_l2(g0["d_densities"], go["d_densities"]) > 10 * GRAD_TOL
    r.close()


def test_aux_backward_without_dl_aux_is_the_plain_backward(c1_scene, oracle32):
    """dl_d_aux = None: d_aux_data is zero and the other groups equal the
    plain backward's (the reference clears the buffer, lib.rs:2080-2090)."""
    sc = c1_scene
    cam = c1_camera(160, 128)
    m = sc["densities"].size
    ad = np.random.default_rng(4).uniform(-1, 1, 2 * m).astype(np.float32)
    r = _renderer(sc, cam, 2, ad)
    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(sc, cam)
    gt = np.random.default_rng(5).uniform(0, 1, (cam.height, cam.width, 3)).astype(np.float32)
    _, dl = oracle32.loss(ref["image"], gt, 1)
    g = r.backward(dl)
    assert g["d_aux_data"].shape == (2 * m,) and not g["d_aux_data"].any()
    go = oracle32.backward(sc, cam, dl, ref)
    for k in ("d_vertices", "d_densities", "d_color_grads", "d_base_colors"):
        assert rel_l2(g[k], go[k]) <= GRAD_TOL, k
    r.close()


def test_aux_backward_two_tet(oracle32):
    """The two-tet shared-face scene (kernel_tests.rs:61-88) with three aux
    channels: every group against the oracle."""
    from rmesh_b200.camera import make_camera

    sc = two_tet_scene()
    cam = make_camera((3.0, 0.4, 1.0), (0.5, 0.4, 0.0), 90.0, 64, 64)
    rng = np.random.default_rng(8)
    ad = rng.uniform(-1, 1, 6).astype(np.float32)
    r = _renderer(sc, cam, 3, ad)
    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(sc, cam, aux=True, aux_data=ad)
    dl = rng.normal(0, 1e-3, (64, 64, 4)).astype(np.float32)
    dl_aux = rng.normal(0, 1e-3, (64, 64, 3)).astype(np.float32)
    g = r.backward(dl, dl_aux)
    go = oracle32.backward(sc, cam, dl, ref, aux_data=ad, dl_aux=dl_aux)
    for k in GROUPS:
        assert rel_l2(g[k], go[k]) <= GRAD_TOL, k
    r.close()
