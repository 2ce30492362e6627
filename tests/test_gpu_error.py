"""Per-tet error statistics (forward_error, crates/rmesh-python/src/lib.rs:1621-1710;
kernel crates/rmesh-error/src/wgsl/error_tiled_compute.wgsl) on the CUDA path
vs the CPU oracle (needs a B200).  The reference accumulates with float
atomics in no fixed order, so sums are compared at relative L2 <= 1e-4 per
statistic; pixel counts and the integer maxima follow per-pixel decisions
and must agree up to the rare pixel at the transmittance cut."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import c1_camera, make_renderer, rel_l2

pytestmark = pytest.mark.gpu

USED = [0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15]


@pytest.mark.parametrize("res,ts", [((256, 256), 12), ((200, 120), 16)])
def test_error_stats_match_oracle(c1_scene, oracle32, res, ts):
    cam = c1_camera(*res)
    r = make_renderer(c1_scene, cam, tile_size=ts)
    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    rng = np.random.default_rng(7)
    n = cam.width * cam.height
    pe = rng.uniform(0, 1, n).astype(np.float32)
    se = rng.uniform(0, 1, n).astype(np.float32)
    err, cnt = r.forward_error(pe, se)
    ref = oracle32.forward_tiled(c1_scene, cam, tile_size=ts)
    e_ref, c_ref = oracle32.error_stats(c1_scene, cam, ref, pe, se, tile_size=ts)
    assert c_ref[:, 0].sum() > 1000
    for k in USED:
        assert rel_l2(err[:, k], e_ref[:, k]) <= 1e-4, k
    assert np.all(err[:, 3:5] == 0.0)
    assert np.abs(cnt[:, 0] - c_ref[:, 0]).sum() <= max(2, c_ref[:, 0].sum() // 10000)
    assert np.all(np.abs(cnt[:, 1] - c_ref[:, 1]) <= np.maximum(2, c_ref[:, 1] // 10000))
    # a second call clears its outputs first (lib.rs:1662-1663)
    err2, cnt2 = r.forward_error(pe, se)
    assert rel_l2(err2, err) <= 1e-6 and np.array_equal(cnt2[:, 0], cnt[:, 0])


def test_error_requires_forward(c1_scene):
    from rmesh_b200 import RMeshError

    cam = c1_camera(64, 64)
    r = make_renderer(c1_scene, cam)
    with pytest.raises(RMeshError):
        r.forward_error(np.zeros(64 * 64, np.float32), np.zeros(64 * 64, np.float32))
