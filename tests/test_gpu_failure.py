"""Failure detection on the GPU without a fault (needs a B200): every wait in
the path's kernels is bounded; a wait on a condition that never resolves
gives up, records an error bit and returns, and the host turns the bit into
RMESH_ERR_TIMEOUT.  The device stays usable afterwards."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import c1_camera, make_renderer

pytestmark = pytest.mark.gpu


def test_bounded_waits_give_up_and_report(c1_scene, oracle32):
    from rmesh_b200 import _lib

    lib = _lib.load()
    bits = np.zeros(2, np.uint32)
    t0 = time.perf_counter()
    assert lib.rmesh_debug_timeouts(bits.ctypes.data) == _lib.RMESH_OK
    assert time.perf_counter() - t0 < 30.0
    assert bits[0] == 2 and bits[1] == 2  # kErrSpinTimeout from the look-back and from the mbarrier
    # the context still works after the timed-out waits
    cam = c1_camera(64, 64)
    r = make_renderer(c1_scene, cam)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(c1_scene, cam)
    assert np.abs(img - ref["image"]).max() <= 1e-4
