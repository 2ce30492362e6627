"""The oracle and the reference-CPU-renderer restatement reproduce the committed
golden fixtures (tests/golden/make_golden.py documents how they were made)."""
from __future__ import annotations

import os

import numpy as np

from conftest import ROOT, known_tet_scene, two_tet_scene

GOLD = os.path.join(ROOT, "tests", "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_known_tet_golden(oracle32):
    from rmesh_b200.camera import make_camera

    g = _load("known_tet.npz")
    f = oracle32.forward_tiled(known_tet_scene(), make_camera((0.0, -2.0, 0.5), (0, 0, 0), 90.0, 64, 64))
    np.testing.assert_array_equal(f["tiles_touched"], g["tiles_touched"])
    np.testing.assert_array_equal(f["key_hi"], g["tiles"])
    np.testing.assert_array_equal(f["vals"], g["tets"])
    np.testing.assert_array_equal(f["ranges"], g["ranges"])
    np.testing.assert_allclose(f["image"], g["image"], atol=1e-6)


def test_two_tet_golden(oracle64):
    from rmesh_b200.camera import make_camera

    g = _load("two_tet.npz")
    sc = {k: (np.asarray(v, np.float64) if v.dtype.kind == "f" else v) for k, v in two_tet_scene().items()}
    cam = make_camera((3.0, 0.4, 1.0), (0.5, 0.4, 0.0), 90.0, 64, 64)
    f = oracle64.forward_tiled(sc, cam)
    loss, dl = oracle64.loss(f["image"], np.full((64, 64, 3), 0.5), 1)
    gr = oracle64.backward(sc, cam, dl, f)
    np.testing.assert_allclose(f["image"], g["image"], atol=1e-12)
    assert abs(loss - float(g["loss"])) < 1e-12
    for k in gr:
        np.testing.assert_allclose(gr[k], g[k], rtol=1e-9, atol=1e-15)
    # the frozen finite differences agree with the analytic density gradient
    np.testing.assert_allclose(g["fd_densities"], g["d_densities"], rtol=1e-3)


def test_four_tet_cpu_renderer_golden():
    from rmesh_b200.camera import make_camera
    from ref_cpu_renderer import cpu_render_scene
    from test_oracle import four_tet_scene

    img = cpu_render_scene(four_tet_scene(), make_camera((2.0, 2.0, 2.0), (0, 0, 0), 90.0, 64, 64))
    np.testing.assert_allclose(img, _load("four_tet_cpu.npz")["image"], atol=1e-6)
