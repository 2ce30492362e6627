"""Camera conventions of the rmeshvk tiled path.

The renderer consumes three flat float32 arrays per view, exactly as the
reference binding does (crates/rmesh-python/src/lib.rs:117-136, 1040-1048):

* ``cam_pos``         [3]  camera position in world space
* ``vp``              [16] view-projection matrix, column-major
* ``c2w_intrinsics``  [16] ``[c2w col0 xyz, 0, col1 xyz, 0, col2 xyz, 0, fx, fy, cx, cy]``

The helpers below build those arrays with the reference's conventions:
left-handed perspective with depth in [0, 1] and look-at with a Z-up world
(crates/rmesh-util/src/camera.rs:103-126), and a pinhole c2w whose columns are
(right, -up, forward) with ``fx = fy = f * H / 2`` and the principal point at
the image centre (crates/rmesh-backward/tests/kernel_tests.rs:44-57).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Camera", "perspective_matrix", "look_at", "make_camera", "orbit_cameras"]


def perspective_matrix(fov_y_rad: float, aspect: float, near: float, far: float) -> np.ndarray:
    """4x4 (row-major math layout) LH perspective, depth in [0,1] (camera.rs:103-111)."""
    f = 1.0 / np.tan(fov_y_rad / 2.0)
    m = np.zeros((4, 4), dtype=np.float64)
    m[0, 0] = f / aspect
    m[1, 1] = f
    m[2, 2] = far / (far - near)
    m[2, 3] = -(far * near) / (far - near)
    m[3, 2] = 1.0
    return m


def look_at(eye, target, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """4x4 view matrix, forward = +Z in view space (camera.rs:114-126)."""
    eye = np.asarray(eye, dtype=np.float64)
    target = np.asarray(target, dtype=np.float64)
    up = np.asarray(up, dtype=np.float64)
    f = target - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.eye(4, dtype=np.float64)
    m[0, :3] = r
    m[1, :3] = u
    m[2, :3] = f
    m[0, 3] = -r.dot(eye)
    m[1, 3] = -u.dot(eye)
    m[2, 3] = -f.dot(eye)
    return m


@dataclass
class Camera:
    """One view: the three flat arrays of the reference API plus its size."""

    cam_pos: np.ndarray  # float32 [3]
    vp: np.ndarray  # float32 [16] column-major
    c2w_intrinsics: np.ndarray  # float32 [16]
    width: int
    height: int

    @property
    def n_pixels(self) -> int:
        return int(self.width) * int(self.height)


def make_camera(eye, target, fov_y_deg: float, width: int, height: int,
                near: float = 0.01, far: float = 100.0, up=(0.0, 0.0, 1.0)) -> Camera:
    """Pinhole camera looking from ``eye`` at ``target`` (kernel_tests.rs:44-57)."""
    fov = np.deg2rad(fov_y_deg)
    proj = perspective_matrix(fov, width / height, near, far)
    view = look_at(eye, target, up)
    vp = proj @ view
    eye = np.asarray(eye, dtype=np.float64)
    f = np.asarray(target, dtype=np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, dtype=np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    c2w = np.stack([r, -u, f], axis=1)  # columns
    f_val = 1.0 / np.tan(fov / 2.0)
    fx = fy = f_val * height / 2.0
    ci = np.zeros(16, dtype=np.float32)
    ci[0:3] = c2w[:, 0]
    ci[4:7] = c2w[:, 1]
    ci[8:11] = c2w[:, 2]
    ci[12:16] = [fx, fy, width / 2.0, height / 2.0]
    return Camera(cam_pos=eye.astype(np.float32),
                  vp=np.ascontiguousarray(vp.T.ravel().astype(np.float32)),
                  c2w_intrinsics=ci, width=int(width), height=int(height))


def orbit_cameras(n: int, seed: int, radius=(2.5, 4.0), resolutions=((512, 512),),
                  fov_y_deg: float = 60.0, target=(0.0, 0.0, 0.0)) -> list:
    """``n`` cameras on a sphere around ``target`` with radius drawn from ``radius``
    and a resolution drawn uniformly from ``resolutions`` (seeded)."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        while True:
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            if abs(d[2]) < 0.9:  # keep away from the look-at singularity at the poles
                break
        rad = rng.uniform(radius[0], radius[1])
        w, h = resolutions[int(rng.integers(len(resolutions)))]
        eye = np.asarray(target, dtype=np.float64) + rad * d
        cams.append(make_camera(eye, target, fov_y_deg, int(w), int(h)))
    return cams
