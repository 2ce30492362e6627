"""numpy restatement of the reference's CPU reference renderer (test infrastructure).

crates/rmesh-render/tests/common/mod.rs:22-351 renders every visible tet for
every pixel, sorted back to front by the circumsphere key, with exact ray-tet
intersection and premultiplied "over" blending -- a different algorithm from the
tiled path (no tiling, no scanline coverage, no culls beyond the frustum).  The
reference compares its GPU tiled image to it with a mean-abs tolerance of 0.02
(single_tet_test.rs:21, multi_tet_test.rs:20); the tests here apply the same
comparison to the CPU oracle, which pins the oracle's rasterizer semantics to
the reference's own independent check.
"""
from __future__ import annotations

import numpy as np

FACES = ((0, 2, 1, 3), (1, 2, 3, 0), (0, 3, 2, 1), (3, 0, 1, 2))


def _ray_dirs(cam) -> np.ndarray:
    """[H, W, 3] unit ray directions (camera.rs:151-175)."""
    ci = np.asarray(cam.c2w_intrinsics, np.float64)
    c2w = np.stack([ci[0:3], ci[4:7], ci[8:11]], axis=1)
    fx, fy, cx, cy = ci[12:16]
    py, px = np.mgrid[0:cam.height, 0:cam.width].astype(np.float64)
    d = np.stack([(px + 0.5 - cx) / fx, (py + 0.5 - cy) / fy, np.ones_like(px)], axis=-1)
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    d = d @ c2w.T
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    return d


def cpu_render_scene(scene: dict, cam, colors=None) -> np.ndarray:
    """[H, W, 4] premultiplied RGBA (common/mod.rs:240-351).  ``colors`` defaults
    to the scene's base colours (the reference harness uses 0.5 for both paths)."""
    v = np.asarray(scene["vertices"], np.float64).reshape(-1, 3)
    t = np.asarray(scene["indices"], np.int64).reshape(-1, 4)
    dens = np.asarray(scene["densities"], np.float64)
    grads = np.asarray(scene["color_grads"], np.float64).reshape(-1, 3)
    col = np.asarray(scene["base_colors"] if colors is None else colors, np.float64).reshape(-1, 3)
    circ = np.asarray(scene["circumdata"], np.float32).reshape(-1, 4)
    cam_pos = np.asarray(cam.cam_pos, np.float64)
    vp = np.asarray(cam.vp, np.float64).reshape(4, 4).T  # column-major -> matrix
    # back-to-front order: ascending ~bits(|C - cam|^2 - r^2) (common/mod.rs:176-200)
    diff = circ[:, :3] - np.asarray(cam.cam_pos, np.float32)
    depth = (np.einsum("ij,ij->i", diff, diff) - circ[:, 3]).astype(np.float32)
    key = ~depth.view(np.uint32)
    order = np.argsort(key, kind="stable")
    # frustum + extent cull (common/mod.rs:280-311)
    vis = np.ones(len(t), bool)
    for i in range(len(t)):
        c = np.c_[v[t[i]], np.ones(4)] @ vp.T
        ndc = c[:, :3] / (c[:, 3:4] + 1e-6)
        mn, mx = ndc.min(0), ndc.max(0)
        if mx[0] < -1 or mn[0] > 1 or mx[1] < -1 or mn[1] > 1 or mn[2] > 1:
            vis[i] = False
        elif (mx[0] - mn[0]) * cam.width * (mx[1] - mn[1]) * cam.height < 1.0:
            vis[i] = False
    d = _ray_dirs(cam)
    acc = np.zeros(d.shape[:2] + (4,))
    for ti in order:
        if not vis[ti]:
            continue
        verts = v[t[ti]]
        num = np.zeros(4)
        nrm = np.zeros((4, 3))
        for f, (a, b, c_, o) in enumerate(FACES):
            n = np.cross(verts[c_] - verts[a], verts[b] - verts[a])
            if n.dot(verts[o] - verts[a]) < 0:
                n = -n
            nrm[f] = n
            num[f] = n.dot(verts[a] - cam_pos)
        den = d @ nrm.T  # [H, W, 4]
        par = np.abs(den) < 1e-20
        valid = ~np.any(par & (num > 0), axis=-1)
        with np.errstate(divide="ignore", invalid="ignore"):
            tt = num / np.where(par, 1.0, den)
        t_min = np.max(np.where((den > 0) & ~par, tt, -np.inf), axis=-1)
        t_max = np.min(np.where((den < 0) & ~par, tt, np.inf), axis=-1)
        dist = np.maximum(t_max - t_min, 0.0)
        od = dens[ti] * dist
        g = grads[ti]
        base = col[ti] + g.dot(cam_pos - verts[0])
        dcdt = d @ g
        with np.errstate(invalid="ignore"):
            cs = np.maximum(base[None, None, :] + (dcdt * t_min)[..., None], 0.0)
            ce = np.maximum(base[None, None, :] + (dcdt * t_max)[..., None], 0.0)
        alpha_t = np.exp(-od)
        with np.errstate(divide="ignore", invalid="ignore"):
            phi = np.where(np.abs(od) < 0.02, 1.0 + od * (-0.5 + od * (1.0 / 6.0 + od * (-1.0 / 24.0))),
                           (1.0 - np.exp(-od)) / od)
        w0 = phi - alpha_t
        w1 = 1.0 - phi
        c = ce * w0[..., None] + cs * w1[..., None]
        a = 1.0 - alpha_t
        c = np.where(valid[..., None] & np.isfinite(c), c, 0.0)
        a = np.where(valid & np.isfinite(a), a, 0.0)
        acc[..., :3] = c + acc[..., :3] * (1.0 - a)[..., None]
        acc[..., 3] = a + acc[..., 3] * (1.0 - a)
    return acc.astype(np.float32)


def compare_images(a, b):
    """(max_diff, mean_diff) over all pixels and channels (common/mod.rs:1637-1660)."""
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(d.max()), float(d.mean())
