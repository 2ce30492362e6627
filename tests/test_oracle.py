"""The CPU oracle pinned to the reference's own known-answer tests and fixtures.

The reference stores no golden files: every check in its test tree is a KAT, a
CPU-vs-GPU comparison against its CPU reference renderer, or a finite-difference
gradient check.  Each is restated here against the oracle (CPU only).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import known_tet_scene, two_tet_scene
from ref_cpu_renderer import compare_images, cpu_render_scene

W = H = 64


def _cam(eye, target, fov=90.0, w=W, h=H):
    from rmesh_b200.camera import make_camera

    return make_camera(eye, target, fov, w, h)


def _random_single_tet(rng, radius):
    """test_util.rs:166-229: random tet, positive orientation, density U[0.5, 5.5),
    colour gradient U[-0.1, 0.1), base colour 0.5 (the reference harness)."""
    from rmesh_b200.scenes import circumspheres

    v = ((rng.random(12) - 0.5) * 2.0 * radius).astype(np.float32)
    p = v.reshape(4, 3).astype(np.float64)
    det = np.dot(p[1] - p[0], np.cross(p[2] - p[0], p[3] - p[0]))
    idx = np.array([0, 1, 3, 2] if det < 0 else [0, 1, 2, 3], np.uint32)
    return {"vertices": v, "indices": idx, "base_colors": np.full(3, 0.5, np.float32),
            "densities": np.array([rng.random() * 5.0 + 0.5], np.float32),
            "color_grads": ((rng.random(3) - 0.5) * 0.2).astype(np.float32),
            "circumdata": circumspheres(v, idx)}


# ---------------------------------------------------------------- KATs
def test_loss_l1_kat(oracle32):
    """kernel_tests.rs:176-305: constant 0.8/0.6/0.4 vs 0.5 -> grad +-1/n_pixels, alpha 0."""
    n = W * H
    rendered = np.tile(np.array([0.8, 0.6, 0.4, 1.0], np.float32), (H, W, 1))
    gt = np.full((H, W, 3), 0.5, np.float32)
    _, dl = oracle32.loss(rendered, gt, 0)
    np.testing.assert_allclose(dl[..., 0], 1.0 / n, atol=1e-5)
    np.testing.assert_allclose(dl[..., 1], 1.0 / n, atol=1e-5)
    np.testing.assert_allclose(dl[..., 2], -1.0 / n, atol=1e-5)
    np.testing.assert_allclose(dl[..., 3], 0.0, atol=1e-5)


def test_loss_l2_value(oracle32):
    """L2 gradient 2(r-gt)/n and the host loss value (kernel_tests.rs:869-878)."""
    rng = np.random.default_rng(3)
    r = rng.uniform(0, 1, (H, W, 4)).astype(np.float32)
    gt = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    loss, dl = oracle32.loss(r, gt, 1)
    diff = r[..., :3].astype(np.float64) - gt
    assert abs(loss - (diff ** 2).sum() / (W * H)) < 1e-9
    np.testing.assert_allclose(dl[..., :3], (2.0 * (r[..., :3] - gt) / np.float32(W * H)), rtol=1e-6)


def test_adam_kat(oracle32):
    """kernel_tests.rs:314-420: params [1,2,3,4], grads [.1,-.2,.3,-.4], lr 0.01, step 1."""
    p = np.array([1, 2, 3, 4], np.float32)
    g = np.array([0.1, -0.2, 0.3, -0.4], np.float32)
    m = np.zeros(4, np.float32)
    v = np.zeros(4, np.float32)
    p0 = p.copy()
    oracle32.adam(p, g, m, v, 1, 0.01)
    assert np.all(np.abs(p - p0) > 1e-6)
    assert np.all(np.sign(p - p0) == -np.sign(g))
    np.testing.assert_allclose(m, 0.1 * g, atol=1e-6)
    # bias-corrected first step moves every parameter by ~lr
    np.testing.assert_allclose(np.abs(p - p0), 0.01, rtol=1e-3)


def test_adam_nan_and_clip(oracle32):
    """adam_compute.wgsl:129-130: NaN gradients count as 0, others clip to +-1e20."""
    p = np.array([1.0, 1.0], np.float32)
    m = np.zeros(2, np.float32)
    v = np.zeros(2, np.float32)
    oracle32.adam(p, np.array([np.nan, np.inf], np.float32), m, v, 1, 0.1)
    assert p[0] == 1.0 and m[0] == 0.0 and np.isfinite(p[1]) and p[1] < 1.0


def test_sort_kat(oracle32):
    """kernel_tests.rs:97-167: 64 random keys sort ascending, values follow their keys."""
    rng = np.random.default_rng(42424242)
    lo = rng.integers(0, 2 ** 32, 64, dtype=np.uint64).astype(np.uint32)
    hi = rng.integers(0, 7, 64).astype(np.uint32)
    vals = np.arange(64, dtype=np.uint32)
    slo, shi, sv = oracle32.sort_pairs(lo, hi, vals, num_tiles=7)
    key = (shi.astype(np.uint64) << 32) | slo
    assert np.all(np.diff(key.astype(np.float64)) >= 0)
    np.testing.assert_array_equal(lo[sv], slo)
    np.testing.assert_array_equal(hi[sv], shi)


def test_sort_is_stable_and_masks_bits(oracle32):
    """drs.rs:23-26: only the low round8(32 + ceil(log2 tiles)) bits are sorted,
    stably -- equal masked keys keep their input order."""
    assert oracle32.sorting_bits(1849) == 48 and oracle32.sorting_bits(2 ** 16 + 1) == 56
    lo = np.array([5, 5, 5, 1], np.uint32)
    hi = np.array([0x10000 + 3, 3, 3, 3], np.uint32)  # bit 48 is outside the sorted bits
    vals = np.array([0, 1, 2, 3], np.uint32)
    _, _, sv = oracle32.sort_pairs(lo, hi, vals, num_tiles=1849)
    np.testing.assert_array_equal(sv, [3, 0, 1, 2])


def test_sentinel_slots(oracle32):
    """tile_fill_compute.wgsl:9-19 + tile_gen_scan_compute.wgsl:190-202: slots a
    tet does not fill keep (0xFFFFFFFF, 0xFFFFFFFF, 0), sort last, and leave the
    last real tile's end unwritten (tile_ranges_compute.wgsl:224-247)."""
    sc = known_tet_scene()
    cam = _cam((0.0, -2.0, 0.5), (0, 0, 0))
    visible, tt, _ = oracle32.project(sc, cam)
    assert visible[0] == 1 and tt[0] > 0
    tt_more = tt + 3  # claim three more tiles than the tet reaches
    lo, hi, vals, emitted = oracle32.emit(sc, cam, visible, tt_more)
    assert emitted == int(tt[0]) and lo.size == int(tt[0]) + 3
    assert np.all(hi[-3:] == 0xFFFFFFFF) and np.all(lo[-3:] == 0xFFFFFFFF) and np.all(vals[-3:] == 0)
    tiles = ((W + 11) // 12) * ((H + 11) // 12)
    slo, shi, sv = oracle32.sort_pairs(lo, hi, vals, tiles)
    assert np.all(shi[-3:] == 0xFFFFFFFF)
    ranges = oracle32.tile_ranges(shi, tiles).reshape(-1, 2)
    last = int(shi[emitted - 1])
    assert ranges[last, 1] == 0  # end never written
    ok = oracle32.tile_ranges(oracle32.sort_pairs(*oracle32.emit(sc, cam, visible, tt)[:3], tiles)[1], tiles)
    assert ok.reshape(-1, 2)[last, 1] == emitted


# ------------------------------------------------------------ camera KATs
def test_camera_cpu_projection():
    """kernel_tests.rs:1547-1612: vp*inv(vp) ~ I, all 4 vertices in NDC, area >= 1 px."""
    sc = known_tet_scene()
    cam = _cam((0.0, -2.0, 0.5), (0, 0, 0))
    vp = cam.vp.reshape(4, 4).T.astype(np.float64)
    np.testing.assert_allclose(vp @ np.linalg.inv(vp), np.eye(4), atol=1e-4)
    pts = np.c_[sc["vertices"].reshape(4, 3), np.ones(4)] @ vp.T
    assert np.all(pts[:, 3] > 0)
    ndc = pts[:, :3] / (pts[:, 3:4] + 1e-6)
    assert np.all(np.abs(ndc[:, :2]) <= 1) and np.all((ndc[:, 2] >= 0) & (ndc[:, 2] <= 1))
    pxy = np.c_[(ndc[:, 0] + 1) * 0.5 * W, (1 - ndc[:, 1]) * 0.5 * H]
    assert np.ptp(pxy[:, 0]) * np.ptp(pxy[:, 1]) >= 1.0


def test_camera_visibility_and_forward(oracle32):
    """kernel_tests.rs:1619-1838: the known tet is visible, touches tiles, and the
    tiled forward (tile size 12) is finite with total alpha > 0.001."""
    sc = known_tet_scene()
    cam = _cam((0.0, -2.0, 0.5), (0, 0, 0))
    f = oracle32.forward_tiled(sc, cam)
    assert f["visible"].sum() == 1 and f["tiles_touched"][0] > 0
    assert np.isfinite(f["image"]).all() and f["image"][..., 3].sum() > 0.001


def test_camera_ray_tet_intersection():
    """kernel_tests.rs:1839-1906: the centre ray hits the known tet in front of the camera."""
    from ref_cpu_renderer import FACES

    sc = known_tet_scene()
    cam_pos = np.array([0.0, -2.0, 0.5])
    v = sc["vertices"].reshape(4, 3).astype(np.float64)
    d = -cam_pos / np.linalg.norm(cam_pos)
    t_in, t_out = -np.inf, np.inf
    for a, b, c, o in FACES:
        n = np.cross(v[c] - v[a], v[b] - v[a])
        if n.dot(v[o] - v[a]) < 0:
            n = -n
        den, num = n.dot(d), n.dot(v[a] - cam_pos)
        if den > 0:
            t_in = max(t_in, num / den)
        elif den < 0:
            t_out = min(t_out, num / den)
    assert 0 < t_in < t_out


# ------------------------------------------- images vs the reference CPU renderer
@pytest.mark.parametrize("offset", [0.1, 1.0, 5.0, 10.0])
def test_single_tet_face_view(oracle32, offset):
    """single_tet_test.rs:85-118: camera in front of face 0 at several offsets,
    oracle tiled image vs CPU reference renderer, mean-abs < 0.02."""
    rng = np.random.default_rng(189710234)
    sc = _random_single_tet(rng, 0.3)
    v = sc["vertices"].reshape(4, 3)[sc["indices"]].astype(np.float64)
    centroid = v.mean(0)
    face_center = (v[0] + v[2] + v[1]) / 3.0
    n = face_center - centroid
    eye = face_center + n / np.linalg.norm(n) * offset
    cam = _cam(eye, centroid)
    img = oracle32.forward_tiled(sc, cam)["image"]
    ref = cpu_render_scene(sc, cam)
    _, mean = compare_images(img, ref)
    assert mean < 0.02, mean


def test_two_tet_outside_view(oracle32):
    """multi_tet_test.rs:131-153 (sorting across tets), mean-abs < 0.02."""
    sc = two_tet_scene()
    sc["base_colors"] = np.full(6, 0.5, np.float32)
    cam = _cam((3.0, 0.4, 1.0), (0.5, 0.4, 0.0))
    img = oracle32.forward_tiled(sc, cam)["image"]
    _, mean = compare_images(img, cpu_render_scene(sc, cam))
    assert mean < 0.02, mean


def four_tet_scene(seed=11):
    from rmesh_b200.scenes import circumspheres

    rng = np.random.default_rng(seed)
    s = 0.5
    v = np.array([0, 0, 0, s, s, s, -s, s, s, -s, -s, s, s, -s, s, s, s, -s, -s, s, -s, -s, -s, -s, s, -s, -s],
                 np.float32)
    idx = np.array([0, 1, 2, 3, 0, 1, 4, 5, 0, 2, 6, 3, 0, 5, 8, 7], np.uint32)
    return {"vertices": v, "indices": idx, "base_colors": np.full(12, 0.5, np.float32),
            "densities": (rng.random(4) * 3.0 + 0.5).astype(np.float32),
            "color_grads": ((rng.random(12) - 0.5) * 0.1).astype(np.float32),
            "circumdata": circumspheres(v, idx)}


# (0, 0, 3) looking at the origin is degenerate with the Z-up look-at, so the
# third viewpoint of multi_tet_test.rs:160-165 is nudged off the axis.
@pytest.mark.parametrize("eye", [(3.0, 0.0, 0.0), (0.0, 3.0, 0.0), (0.0, 0.05, 3.0), (2.0, 2.0, 2.0)])
def test_four_tet_multi_angle(oracle32, eye):
    """multi_tet_test.rs:157-183, mean-abs < 0.02."""
    sc = four_tet_scene()
    cam = _cam(eye, (0, 0, 0))
    img = oracle32.forward_tiled(sc, cam)["image"]
    _, mean = compare_images(img, cpu_render_scene(sc, cam))
    assert mean < 0.02, mean


def test_tet_at_boundary(oracle32):
    """cross_renderer_test.rs:766-810: the known tet at the edge of the frame;
    tiled vs the CPU renderer max-abs < 0.002, mean-abs < 0.02."""
    sc = known_tet_scene()
    cam = _cam((3.0, 1.5, 0.0), (0.0, 1.5, 0.0))
    img = oracle32.forward_tiled(sc, cam)["image"]
    mx, mean = compare_images(img, cpu_render_scene(sc, cam))
    assert img[..., 3].max() > 0.01
    assert mx < 0.002 and mean < 0.02, (mx, mean)


def test_tet_behind_camera(oracle32):
    """cross_renderer_test.rs:812-850: camera looking away from the tet: the
    alpha sum stays below 0.01 (here exactly zero: nothing is binned)."""
    sc = known_tet_scene()
    cam = _cam((3.0, 0.0, 0.0), (10.0, 0.0, 0.0))
    f = oracle32.forward_tiled(sc, cam)
    assert f["P"] == 0 and f["image"][..., 3].sum() < 0.01
    assert cpu_render_scene(sc, cam)[..., 3].sum() < 0.01


def test_distant_tet(oracle32):
    """cross_renderer_test.rs:853-888: at distance 50 the tet covers a pixel
    or less; tiled vs the CPU renderer mean-abs < 0.01."""
    sc = known_tet_scene()
    cam = _cam((50.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    img = oracle32.forward_tiled(sc, cam)["image"]
    _, mean = compare_images(img, cpu_render_scene(sc, cam))
    assert mean < 0.01, mean


def test_center_pixel(oracle32):
    """cross_renderer_test.rs:893-981: the centre pixel of the known tet seen
    from (3, 0, 0) has alpha > 0.01, non-negative premultiplied colour, and
    matches the CPU renderer within 0.01 per channel."""
    sc = known_tet_scene()
    cam = _cam((3.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    img = oracle32.forward_tiled(sc, cam)["image"]
    ref = cpu_render_scene(sc, cam)
    px, want = img[H // 2, W // 2], ref[H // 2, W // 2]
    assert want[3] > 0.01 and np.all(want[:3] >= -1e-6)
    assert np.all(np.abs(px - want) < 0.01), (px, want)


def test_tiled_forward_multi_scene_finite(oracle32, c1_scene):
    """kernel_tests.rs:549-718: a many-tet tiled forward is finite and non-zero."""
    from conftest import c1_camera

    f = oracle32.forward_tiled(c1_scene, c1_camera(128, 128))
    assert np.isfinite(f["image"]).all() and f["image"][..., 3].max() > 0.1


# ---------------------------------------------------------- gradients (FD)
def _fd_loss(o, sc, cam, gt, loss_type=1):
    f = o.forward_tiled(sc, cam)
    val, _ = o.loss(f["image"], gt, loss_type)
    return val


def test_two_tet_fd_gradients(oracle64):
    """kernel_tests.rs:733-1168: two-tet scene, 64x64, L2 vs gray 0.5; central FD
    (eps 1e-3, colour gradients 1e-2) with circumspheres recomputed per perturbation;
    rel_tol 0.10, abs_tol 5e-5.  Evaluated in float64."""
    from rmesh_b200.scenes import circumspheres

    sc = {k: (np.asarray(v, np.float64) if v.dtype.kind == "f" else v) for k, v in two_tet_scene().items()}
    cam = _cam((3.0, 0.4, 1.0), (0.5, 0.4, 0.0))
    gt = np.full((H, W, 3), 0.5)
    f = oracle64.forward_tiled(sc, cam)
    _, dl = oracle64.loss(f["image"], gt, 1)
    g = oracle64.backward(sc, cam, dl, f)
    fails = []
    for key, gkey, eps in (("densities", "d_densities", 1e-3), ("vertices", "d_vertices", 1e-3),
                           ("color_grads", "d_color_grads", 1e-2), ("base_colors", "d_base_colors", 1e-3)):
        for i in range(sc[key].size):
            vals = []
            for s in (+1, -1):
                sp = {k: v.copy() for k, v in sc.items()}
                sp[key][i] += s * eps
                if key == "vertices":
                    sp["circumdata"] = circumspheres(sp["vertices"], sp["indices"]).astype(np.float64)
                vals.append(_fd_loss(oracle64, sp, cam, gt))
            num = (vals[0] - vals[1]) / (2 * eps)
            ana = g[gkey][i]
            abs_err = abs(ana - num)
            rel = abs_err / max(abs(ana), abs(num), 1e-7)
            if rel > 0.10 and abs_err > 5e-5 and (abs(ana) > 1e-7 or abs(num) > 1e-7):
                fails.append((key, i, ana, num, rel))
    assert not fails, fails


def test_aux_channel_fd_gradients(oracle64):
    """The adjoint of the custom aux channels (orc_backward_aux): the forward
    composites aux += T alpha a[t] per item (rasterize_compute.wgsl:458-462).
    For the linear functional L = sum(dl_img * image) + sum(dl_aux * aux) on
    the two-tet scene, every gradient group (aux data, densities, vertices,
    colour gradients, base colours) matches float64 central differences."""
    from rmesh_b200.scenes import circumspheres

    sc = {k: (np.asarray(v, np.float64) if v.dtype.kind == "f" else v) for k, v in two_tet_scene().items()}
    cam = _cam((3.0, 0.4, 1.0), (0.5, 0.4, 0.0))
    rng = np.random.default_rng(11)
    aux_dim = 3
    ad = rng.uniform(-1, 1, 2 * aux_dim)
    dl_img = rng.normal(0, 1e-3, (H, W, 4))
    dl_aux = rng.normal(0, 1e-3, (H, W, aux_dim))

    def objective(s, a):
        f = oracle64.forward_tiled(s, cam, aux=True, aux_data=a)
        return float(np.sum(dl_img * f["image"]) + np.sum(dl_aux * f["aux"][..., 8:]))

    f = oracle64.forward_tiled(sc, cam, aux=True, aux_data=ad)
    assert np.abs(f["aux"][..., 8:]).max() > 0.05
    g = oracle64.backward(sc, cam, dl_img, f, aux_data=ad, dl_aux=dl_aux)
    g0 = oracle64.backward(sc, cam, dl_img, f)
    # the aux channels change the optical-depth gradients
    assert np.abs(g["d_densities"] - g0["d_densities"]).max() > 1e-6
    fails = []
    cases = [("aux", "d_aux_data", 1e-4)] + [(k, gk, 1e-4) for k, gk in
                                             (("densities", "d_densities"), ("vertices", "d_vertices"),
                                              ("color_grads", "d_color_grads"), ("base_colors", "d_base_colors"))]
    for key, gkey, eps in cases:
        n = ad.size if key == "aux" else sc[key].size
        for i in range(n):
            vals = []
            for sgn in (+1, -1):
                sp = {k: v.copy() for k, v in sc.items()}
                a = ad.copy()
                if key == "aux":
                    a[i] += sgn * eps
                else:
                    sp[key][i] += sgn * eps
                    if key == "vertices":
                        sp["circumdata"] = circumspheres(sp["vertices"], sp["indices"]).astype(np.float64)
                vals.append(objective(sp, a))
            num = (vals[0] - vals[1]) / (2 * eps)
            ana = g[gkey][i]
            abs_err = abs(ana - num)
            rel = abs_err / max(abs(ana), abs(num), 1e-9)
            if rel > 1e-3 and abs_err > 1e-8:
                fails.append((key, i, ana, num, rel))
    assert not fails, fails


def test_single_tet_python_fd(oracle64):
    """crates/rmesh-python/tests/test_autograd.py:14-250: numpy RandomState(42)
    single tet, 32x32, camera at distance 1 (GS convention, fov 45), loss
    0.5*sum((rgb - 0)^2), eps 1e-3, per-element rel_err < 0.1."""
    from rmesh_b200.camera import Camera

    rs = np.random.RandomState(42)
    radius = 0.6
    verts = (rs.rand(4, 3).astype(np.float32) - 0.5) * 2.0 * radius
    v0, v1, v2, v3 = verts
    det = np.dot(v1 - v0, np.cross(v2 - v0, v3 - v0))
    indices = np.array([0, 1, 3, 2] if det < 0 else [0, 1, 2, 3], np.uint32)
    base_colors = (rs.rand(3).astype(np.float32) * 2.0 - 1.0)
    densities = np.array([rs.rand() * 5.0 + 0.5], np.float32)
    color_grads = ((rs.rand(3).astype(np.float32) - 0.5) * 0.2)
    from rmesh_b200.scenes import circumspheres

    sc = {"vertices": verts.ravel().astype(np.float64), "indices": indices,
          "base_colors": base_colors.astype(np.float64), "densities": densities.astype(np.float64),
          "color_grads": color_grads.astype(np.float64),
          "circumdata": circumspheres(verts.ravel(), indices).astype(np.float64)}
    Wp = Hp = 32
    d = 1.0
    R = np.array([[1, 0, 0], [0, -1, 0], [0, 0, -1]], np.float64)
    Rt = np.eye(4)
    Rt[:3, :3] = R.T
    Rt[:3, 3] = -R @ np.array([0, 0, d])
    fov = 45.0 * np.pi / 180.0
    f_val = 1.0 / np.tan(fov / 2.0)
    fx = f_val * Wp / 2.0
    fy = f_val * Hp / 2.0
    proj = np.zeros((4, 4))
    proj[0, 0] = 2 * fx / Wp
    proj[0, 2] = 2 * (Wp / 2) / Wp - 1
    proj[1, 1] = -2 * fy / Hp
    proj[1, 2] = 1 - 2 * (Hp / 2) / Hp
    proj[3, 2] = 1.0
    vp = (Rt.T @ proj.T).ravel().astype(np.float32)  # test_autograd.py:104 (row-vector convention)
    ci = np.zeros(16, np.float32)
    ci[0:3], ci[4:7], ci[8:11] = R.T[:, 0], R.T[:, 1], R.T[:, 2]
    ci[12:16] = [fx, fy, Wp / 2, Hp / 2]
    cam = Camera(np.array([0, 0, d], np.float32), vp, ci, Wp, Hp)
    gt = np.zeros((Hp, Wp, 3))

    def loss(s):
        img = oracle64.forward_tiled(s, cam)["image"][..., :3]
        return 0.5 * float(((img - gt) ** 2).sum())

    f = oracle64.forward_tiled(sc, cam)
    dl = np.zeros((Hp, Wp, 4))
    dl[..., :3] = f["image"][..., :3] - gt
    g = oracle64.backward(sc, cam, dl, f)
    assert f["image"][..., 3].sum() > 1.0
    fails = []
    eps = 1e-3
    for key, gkey in (("base_colors", "d_base_colors"), ("densities", "d_densities"),
                      ("color_grads", "d_color_grads"), ("vertices", "d_vertices")):
        for i in range(sc[key].size):
            sp, sm = {k: v.copy() for k, v in sc.items()}, {k: v.copy() for k, v in sc.items()}
            sp[key][i] += eps
            sm[key][i] -= eps
            num = (loss(sp) - loss(sm)) / (2 * eps)
            a = g[gkey][i]
            rel = abs(a - num) / max(abs(a), abs(num), 1e-7)
            if rel >= 0.1:
                fails.append((key, i, a, num, rel))
    assert not fails, fails


def test_single_tet_loss_decreases():
    """kernel_tests.rs:1181-1510: one tet, black target, L2, 200 Adam steps with
    lr 0.1 on densities and colour gradients (vertices frozen): the loss falls
    below 1% of its start and already drops within 10 steps."""
    from oracle import OracleTrainer

    rng = np.random.default_rng(42424242)
    sc = _random_single_tet(rng, 0.6)
    v = sc["vertices"].reshape(4, 3)[sc["indices"]].astype(np.float64)
    centroid = v.mean(0)
    cam = _cam(centroid + np.array([1.0, 0.0, 0.0]), centroid)
    tr = OracleTrainer(sc)
    gt = np.zeros((H, W, 3), np.float32)
    losses = [tr.train_step(cam, gt, 0.0, 0.1, 0.1, 1)[0] for _ in range(200)]
    assert losses[0] > 0
    assert losses[9] < losses[0]
    assert losses[-1] < 0.01 * losses[0], (losses[0], losses[-1])


def test_trainer_views_step_is_the_sum_of_single_view_gradients():
    """The multi-view step: one view equals the single-view train_step; two
    views move the parameters as one Adam step on the summed gradients."""
    from oracle import OracleTrainer

    sc = _sh_scene(seed=5, points=40)
    rng = np.random.default_rng(6)
    cams = [_cam(np.array(e), np.zeros(3)) for e in ((2.2, 0.3, 0.4), (-0.5, 2.0, 1.0))]
    gts = [rng.uniform(0, 1, (H, W, 3)).astype(np.float32) for _ in cams]
    lrs = (1e-3, 1e-2, 1e-2)
    a, b = OracleTrainer(sc, use_sh=True), OracleTrainer(sc, use_sh=True)
    la = a.train_step_views(cams[:1], gts[:1], *lrs, 1, lr_sh=1e-2)
    lb = b.train_step(cams[0], gts[0], *lrs, 1, lr_sh=1e-2)[0]
    assert la[0] == lb
    for k in ("vertices", "densities", "color_grads"):
        np.testing.assert_array_equal(a.scene[k], b.scene[k])
    np.testing.assert_array_equal(a.sh, b.sh)

    c, d = OracleTrainer(sc, use_sh=True), OracleTrainer(sc, use_sh=True)
    lc = c.train_step_views(cams, gts, *lrs, 1, lr_sh=1e-2)
    g = [d._view_grads(cam, gt, 1, 1)[2] for cam, gt in zip(cams, gts)]
    d._adam_all({k: g[0][k] + g[1][k] for k in g[0]}, *lrs, 1e-2)
    assert lc.shape == (2,) and np.all(lc > 0)
    for k in ("vertices", "densities", "color_grads"):
        np.testing.assert_array_equal(c.scene[k], d.scene[k])
    assert np.any(c.scene["densities"] != sc["densities"])


def _sh_scene(seed=3, points=60, degree=3):
    from rmesh_b200.scenes import make_scene, uniform_cloud

    rng = np.random.default_rng(seed)
    sc = make_scene(uniform_cloud(points, rng, -0.6, 0.6), rng, sh_degree=degree)
    return sc


def test_sh_degree0_colour_is_softplus_of_dc(oracle32):
    """project_compute.wgsl:264-318 at degree 0: colour = softplus(C0*sh0 + 0.5 +
    dot(g, v0 - centroid)) per channel, with the f16-rounded coefficient."""
    from rmesh_b200.scenes import SH_C0

    sc = _sh_scene(degree=0)
    cam = _cam((1.8, -1.2, 0.9), (0, 0, 0), 60.0)
    shv = oracle32.sh_values(sc["sh_coeffs"])
    vis, _, col = oracle32.project(sc, cam, 12, sh=shv, sh_degree=0)
    v = sc["vertices"].reshape(-1, 3).astype(np.float64)
    t = sc["indices"].reshape(-1, 4)
    cen = v[t].mean(axis=1)
    off = np.einsum("ij,ij->i", sc["color_grads"].reshape(-1, 3), v[t[:, 0]] - cen)
    rgb = SH_C0 * shv.reshape(-1, 3).astype(np.float64) + 0.5 + off[:, None]
    want = np.where(rgb * 10 > 20, rgb, 0.1 * np.log1p(np.exp(10 * rgb)))
    m = vis.astype(bool)
    assert m.sum() > 20
    np.testing.assert_allclose(col.reshape(-1, 3)[m], want[m], rtol=2e-5, atol=2e-6)


def test_sh_fd_gradients(oracle64):
    """Adjoint of the SH colour (no reference counterpart): central finite
    differences in float64, step 1e-4, on sampled coefficients, colour gradients,
    densities and vertices of a degree-3 scene (the gradient check of the
    10k-point degree-3 configuration, at a size the oracle finishes quickly)."""
    sc = {k: (np.asarray(v, np.float64) if isinstance(v, np.ndarray) and v.dtype.kind == "f" else v)
          for k, v in _sh_scene().items()}
    deg = sc["sh_degree"]
    cam = _cam((1.9, -1.1, 0.8), (0, 0, 0), 60.0)
    gt = np.random.default_rng(8).uniform(0, 1, (H, W, 3))
    sh = oracle64.sh_values(sc["sh_coeffs"], f16=False)

    def loss_of(scene, shv):
        f = oracle64.forward_tiled(scene, cam, sh=shv, sh_degree=deg)
        return oracle64.loss(f["image"], gt, 1)[0]

    f = oracle64.forward_tiled(sc, cam, sh=sh, sh_degree=deg)
    _, dl = oracle64.loss(f["image"], gt, 1)
    g = oracle64.backward(sc, cam, dl, f, sh=sh, sh_degree=deg)
    assert np.abs(g["d_base_colors"]).max() == 0.0
    rng = np.random.default_rng(11)
    eps = 1e-4
    fails, checked = [], 0
    for key, gkey, n in (("sh", "d_sh", 60), ("color_grads", "d_color_grads", 30), ("densities", "d_densities", 20),
                         ("vertices", "d_vertices", 30)):
        arr = sh if key == "sh" else sc[key]
        # sample among parameters with a non-negligible gradient so the check has teeth
        cand = np.nonzero(np.abs(g[gkey]) > 1e-6)[0]
        assert cand.size >= 5, key
        for i in rng.choice(cand, size=min(n, cand.size), replace=False):
            vals = []
            for sgn in (+1, -1):
                a2 = arr.copy()
                a2[i] += sgn * eps
                if key == "sh":
                    vals.append(loss_of(sc, a2))
                else:
                    sp = dict(sc)
                    sp[key] = a2
                    vals.append(loss_of(sp, sh))
            num = (vals[0] - vals[1]) / (2 * eps)
            ana = g[gkey][i]
            err = abs(ana - num)
            tol = 1e-3 if key in ("sh", "color_grads") else 0.10  # vertices/densities: pixel coverage steps
            if err > tol * max(abs(ana), abs(num)) and err > 1e-7:
                fails.append((key, int(i), float(ana), float(num)))
            checked += 1
    assert checked >= 100
    assert len(fails) <= 2, fails  # a vertex step may cross a pixel-coverage edge


def test_c2_fd_gradients_200_per_group(oracle64):
    """The 10,000-point degree-3 configuration's gradient check: central finite
    differences in float64, step 1e-4, on 200 sampled parameters per group
    (SH coefficients, colour gradients, densities, vertices), against the
    adjoint (tile walk + SH colour adjoint).  Parameters are drawn among those
    with a non-zero gradient so each sample tests something; SH values are the
    f16-rounded ones the renderer reads, perturbed in float64."""
    from rmesh_b200.scenes import scene_for_config

    sc = {k: (np.asarray(v, np.float64) if isinstance(v, np.ndarray) and v.dtype.kind == "f" else v)
          for k, v in scene_for_config("c2").items()}
    deg = sc["sh_degree"]
    cam = _cam((1.2, -2.5, 1.1), (0, 0, 0), 50.0, 64, 64)
    gt = np.random.default_rng(8).uniform(0, 1, (64, 64, 3))
    sh = oracle64.sh_values(sc["sh_coeffs"]).astype(np.float64)

    def loss_of(scene, shv):
        f = oracle64.forward_tiled(scene, cam, sh=shv, sh_degree=deg)
        return oracle64.loss(f["image"], gt, 1)[0]

    f = oracle64.forward_tiled(sc, cam, sh=sh, sh_degree=deg)
    _, dl = oracle64.loss(f["image"], gt, 1)
    g = oracle64.backward(sc, cam, dl, f, sh=sh, sh_degree=deg, threads=0)
    rng = np.random.default_rng(13)
    eps = 1e-4
    # per sample: relative error <= tol or absolute <= 1e-8; the loss has kinks
    # (ReLU'd segment colours, pixel coverage for vertices) where a central
    # difference straddles a non-smooth point, so a few samples may miss
    for key, gkey, tol, min_pass in (("sh", "d_sh", 1e-3, 0.97), ("color_grads", "d_color_grads", 1e-3, 0.97),
                                     ("densities", "d_densities", 1e-3, 0.95), ("vertices", "d_vertices", 1e-2, 0.9)):
        arr = sh if key == "sh" else sc[key]
        cand = np.nonzero(np.abs(g[gkey]) > 1e-7)[0]
        idx = rng.choice(cand, size=min(200, cand.size), replace=False)
        num = np.empty(idx.size)
        for j, i in enumerate(idx):
            vals = []
            for sgn in (+1, -1):
                a2 = arr.copy()
                a2[i] += sgn * eps
                vals.append(loss_of(sc, a2) if key == "sh" else loss_of({**sc, key: a2}, sh))
            num[j] = (vals[0] - vals[1]) / (2 * eps)
        ana = g[gkey][idx]
        err = np.abs(ana - num)
        ok = (err <= tol * np.maximum(np.abs(ana), np.abs(num))) | (err <= 1e-8)
        assert idx.size >= 100 and ok.mean() >= min_pass, (key, ok.mean(), float(np.median(err / np.abs(num))))


def test_grid_scene_structure():
    """grid_scene restates the reference's grid layout: n^3 vertices, five
    tets per cell over the cell's eight corners, every tet non-degenerate."""
    from rmesh_b200.scenes import grid_scene

    sc = grid_scene(4, np.random.default_rng(1), jitter=0.0)
    v = sc["vertices"].reshape(-1, 3).astype(np.float64)
    idx = sc["indices"].reshape(-1, 4)
    assert v.shape == (64, 3) and idx.shape == (27 * 5, 4)
    assert sc["circumdata"].size == 4 * idx.shape[0]
    a, b, c, d = (v[idx[:, k]] for k in range(4))
    vol = np.abs(np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)) / 6.0
    step = 1.0 / 3.0
    # four corner tets of volume step^3/6 and the central one of step^3/3 per cell
    np.testing.assert_allclose(np.sort(vol.reshape(27, 5), axis=1),
                               np.tile([step ** 3 / 6] * 4 + [step ** 3 / 3], (27, 1)), rtol=1e-5)
