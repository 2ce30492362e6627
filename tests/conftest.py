"""Shared fixtures: seeded scenes, reference-convention cameras, the CPU oracle."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def known_tet_scene():
    """Regular tet inside the unit cube, density 3, zero colour gradient
    (crates/rmesh-backward/tests/kernel_tests.rs:1516-1545)."""
    from rmesh_b200.scenes import circumspheres

    v = np.array([0.5, 0.5, 0.5, -0.5, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5, -0.5, -0.5], np.float32)
    idx = np.array([0, 1, 2, 3], np.uint32)
    return {"vertices": v, "indices": idx, "base_colors": np.full(3, 0.5, np.float32),
            "densities": np.array([3.0], np.float32), "color_grads": np.zeros(3, np.float32),
            "circumdata": circumspheres(v, idx)}


def two_tet_scene(seed=7):
    """Two tets sharing a face (kernel_tests.rs:61-88), parameters from a seeded rng."""
    from rmesh_b200.scenes import circumspheres

    rng = np.random.default_rng(seed)
    v = np.array([0, 0, 0, 1, 0, 0, 0.5, 1, 0, 0.5, 0.3, 0.8, 0.5, 0.3, -0.8], np.float32)
    idx = np.array([0, 1, 2, 3, 0, 2, 1, 4], np.uint32)
    return {"vertices": v, "indices": idx, "base_colors": rng.uniform(0.2, 0.8, 6).astype(np.float32),
            "densities": (rng.random(2) * 3.0 + 0.5).astype(np.float32),
            "color_grads": ((rng.random(6) - 0.5) * 0.1).astype(np.float32),
            "circumdata": circumspheres(v, idx)}


def c1_camera(width=512, height=512):
    from rmesh_b200.camera import make_camera

    d = np.array([0.6, -0.8, 0.35])
    return make_camera(3.0 * d / np.linalg.norm(d), (0, 0, 0), 60.0, width, height)


@pytest.fixture(scope="session")
def c1_scene():
    from rmesh_b200.scenes import scene_for_config

    return scene_for_config("c1")


@pytest.fixture(scope="session")
def c2_scene():
    """10,000-point 8-component GMM Delaunay mesh with degree-3 SH colours."""
    from rmesh_b200.scenes import scene_for_config

    return scene_for_config("c2")


@pytest.fixture(scope="session")
def oracle32():
    from oracle import Oracle

    return Oracle("f32")


@pytest.fixture(scope="session")
def oracle64():
    from oracle import Oracle

    return Oracle("f64")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def make_renderer(scene, cam, tile_size=12, sh=False):
    """Renderer over a scene dict; sh=True colours it by its SH coefficients."""
    from rmesh_b200 import RMeshRenderer

    kw = dict(sh_coeffs=scene["sh_coeffs"], sh_degree=scene["sh_degree"]) if sh else {}
    return RMeshRenderer(scene["vertices"], scene["indices"], scene["base_colors"], scene["densities"],
                         scene["color_grads"], scene["circumdata"], cam.width, cam.height, tile_size=tile_size, **kw)
