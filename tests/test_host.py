"""Host-side logic without a GPU: camera conventions, scene generation,
circumspheres, view sharding, benchmark accounting."""
from __future__ import annotations

import numpy as np
import pytest


def test_make_camera_matches_reference_conventions():
    """kernel_tests.rs:44-57 / camera.rs:103-126: fx = fy = f*H/2, principal point
    at the centre, c2w columns (right, -up, forward), LH depth in [0, 1]."""
    from rmesh_b200.camera import make_camera

    cam = make_camera((3.0, 0.4, 1.0), (0.5, 0.4, 0.0), 90.0, 64, 48)
    ci = cam.c2w_intrinsics
    f_val = 1.0 / np.tan(np.pi / 4)
    np.testing.assert_allclose(ci[12:16], [f_val * 24, f_val * 24, 32, 24], rtol=1e-6)
    c2w = np.stack([ci[0:3], ci[4:7], ci[8:11]], axis=1)
    np.testing.assert_allclose(c2w.T @ c2w, np.eye(3), atol=1e-6)
    fwd = c2w[:, 2]
    np.testing.assert_allclose(fwd, np.array([-2.5, 0.0, -1.0]) / np.linalg.norm([-2.5, 0, -1]), atol=1e-6)
    vp = cam.vp.reshape(4, 4).T.astype(np.float64)
    p = vp @ np.r_[0.5, 0.4, 0.0, 1.0]
    assert p[3] > 0 and abs(p[0] / p[3]) < 1e-5 and abs(p[1] / p[3]) < 1e-5 and 0 < p[2] / p[3] < 1
    # the pixel-centre ray through the principal point is the forward axis
    d = np.array([(32 + 0.5 - 32) / ci[12], (24 + 0.5 - 24) / ci[13], 1.0])
    d = c2w @ (d / np.linalg.norm(d))
    assert np.dot(d, fwd) > 0.999


def test_circumspheres_are_equidistant():
    from rmesh_b200.scenes import circumspheres

    rng = np.random.default_rng(0)
    v = rng.normal(size=(40, 3)).astype(np.float32)
    idx = rng.permutation(40)[:40].reshape(10, 4).astype(np.uint32)
    c = circumspheres(v.ravel(), idx.ravel()).reshape(-1, 4).astype(np.float64)
    for t in range(10):
        d2 = ((v[idx[t]].astype(np.float64) - c[t, :3]) ** 2).sum(1)
        np.testing.assert_allclose(d2, c[t, 3], rtol=1e-3)


def test_circumsphere_degenerate_guard():
    """test_autograd.py:25-27: |denom| < 1e-12 -> denom = 1 (finite output)."""
    from rmesh_b200.scenes import circumspheres

    v = np.zeros(12, np.float32)
    c = circumspheres(v, np.arange(4, dtype=np.uint32))
    assert np.isfinite(c).all()


def test_scene_for_config_c1():
    from rmesh_b200.scenes import scene_for_config

    sc = scene_for_config("c1")
    assert sc["vertices"].size == 3 * 2000
    m = sc["indices"].size // 4
    assert 11000 < m < 15000  # ~13k tets
    assert sc["densities"].min() > 0 and sc["circumdata"].size == 4 * m
    assert sc["indices"].max() < 2000


def test_orbit_cameras_resolutions_and_radius():
    from rmesh_b200.camera import orbit_cameras

    res = ((256, 256), (512, 512), (800, 600), (1024, 1024))
    cams = orbit_cameras(16, seed=1, radius=(2.5, 4.0), resolutions=res)
    for c in cams:
        assert (c.width, c.height) in res
        assert 2.5 <= np.linalg.norm(c.cam_pos) <= 4.0


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_views_partition(world):
    from rmesh_b200.dp import shard_views

    got = sorted(i for r in range(world) for i in shard_views(16, world, r))
    assert got == list(range(16))


def test_bench_accounting():
    import bench

    assert bench.algorithmic_bytes(10, 100, 5, 7) == 2 * 10 * 84 + 12 * 100 + 80 * 7
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
