"""Edge cases of the CUDA path vs the oracle (needs a B200): a view that sees
nothing, a camera inside the mesh (negative depth keys, vertices behind the
camera), a multi-view step whose tiles exceed 2^16 in total, pair-buffer
overflow, tile lists of thousands of tets, the reference's grid mesh,
its cross-renderer cameras, and tets large enough that a batch's covered
pixels exceed the kernel's sub-batch capacity."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import make_renderer, rel_l2

pytestmark = pytest.mark.gpu


def test_view_that_sees_nothing(c1_scene, oracle32):
    from rmesh_b200.camera import make_camera

    cam = make_camera((0.0, -6.0, 0.0), (0.0, -20.0, 0.0), 40.0, 96, 64)  # looking away from the mesh
    assert np.isfinite(cam.vp).all()
    r = make_renderer(c1_scene, cam)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(c1_scene, cam)
    assert ref["P"] == 0 and r.info().n_pairs_last == 0
    assert np.all(img == 0.0) and np.all(ref["image"] == 0.0)
    g = r.backward(np.ones((64, 96, 4), np.float32))
    assert all(np.all(v == 0.0) for v in g.values())
    gt = np.full((64, 96, 3), 0.5, np.float32)
    loss = r.train_step(cam.cam_pos, cam.vp, cam.c2w_intrinsics, gt, 1e-4, 1e-2, 1e-3, 1)
    assert abs(loss - 3 * 0.25) < 1e-6
    np.testing.assert_array_equal(r.get_params()["vertices"], c1_scene["vertices"])


def test_camera_inside_the_mesh(c1_scene, oracle32):
    """Tets around the eye have vertices behind the camera (no tiles) and
    circumspheres containing it (negative depth keys, which sort first)."""
    from rmesh_b200.camera import make_camera

    cam = make_camera((0.05, -0.1, 0.02), (1.0, 0.3, 0.2), 70.0, 160, 120)
    r = make_renderer(c1_scene, cam)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(c1_scene, cam)
    assert ref["P"] > 0
    np.testing.assert_array_equal(r.debug_tiles_touched(), np.where(ref["visible"] > 0, ref["tiles_touched"], 0))
    tiles, tets = r.debug_pairs()
    np.testing.assert_array_equal(tiles, ref["key_hi"])
    np.testing.assert_array_equal(tets, ref["vals"])
    assert np.abs(img - ref["image"]).max() <= 1e-4
    gt = np.random.default_rng(3).uniform(0, 1, (120, 160, 3)).astype(np.float32)
    _, dl = oracle32.loss(ref["image"], gt, 1)
    g = r.backward(dl)
    go = oracle32.backward(c1_scene, cam, dl, ref)
    for k in go:
        assert rel_l2(g[k], go[k]) <= 1e-3, k


def test_many_tiles_batched_step(c1_scene, oracle32):
    """8 views of 1024x1024 (59,168 tiles of 12x12... times 8 = 473k > 2^16):
    the batched and graph steps' per-view losses equal the oracle's."""
    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(8, seed=12, radius=(2.6, 3.4), resolutions=((1024, 1024),))
    rng = np.random.default_rng(9)
    gts = [rng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    want = []
    for c, g in zip(cams, gts):
        f = oracle32.forward_tiled(c1_scene, c)
        want.append(oracle32.loss(f["image"], g, 1)[0])
    for mode in ("batched", "graph"):
        r = make_renderer(c1_scene, cams[0])
        losses = r.train_step_views(cams, gts, 0.0, 0.0, 0.0, 1, mode=mode)
        np.testing.assert_allclose(losses, want, rtol=1e-4)
        assert r.info().n_views_last == 8


def test_pair_buffer_overflow_grows_and_retries(oracle32):
    """One tet filling 16 views of 1400x1400: 119,158 (tile, tet) pairs in
    total overflow the initial 65,536-slot pair buffer; the step grows the
    buffer and redoes the run inside the same call (no error reaches the
    caller), the per-view losses equal the oracle's, and a graph-mode step
    after the growth (new buffers, new capture) agrees as well."""
    from conftest import known_tet_scene

    from rmesh_b200.camera import make_camera

    sc = known_tet_scene()
    n = 16
    i = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * i / n)
    th = np.pi * (1 + 5 ** 0.5) * i
    dirs = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)
    cams = [make_camera(tuple(1.6 * d), (0.0, 0.0, 0.0), 45.0, 1400, 1400) for d in dirs]
    rng = np.random.default_rng(17)
    gts = [rng.uniform(0, 1, (1400, 1400, 3)).astype(np.float32) for _ in cams]
    want, total = [], 0
    for c, g in zip(cams, gts):
        f = oracle32.forward_tiled(sc, c)
        total += int(f["P"])
        want.append(oracle32.loss(f["image"], g, 1)[0])
    assert total > 65536
    r = make_renderer(sc, cams[0])
    assert r.info().pair_capacity <= 65536 or r.info().pair_capacity == 0
    for mode in ("batched", "graph", "graph"):
        losses = r.train_step_views(cams, gts, 0.0, 0.0, 0.0, 1, mode=mode)
        np.testing.assert_allclose(losses, want, rtol=1e-4)
        assert r.info().n_pairs_last == total
    assert r.info().pair_capacity >= total
    r.close()


def test_long_tile_lists(c2_scene):
    """65k tets seen at 48x48 (16 tiles of 12x12): each tile's list holds
    thousands of tets (hundreds of 32-tet batches, each with its span records
    bulk-copied beside its tet records, the forward stopping at the
    transmittance cut-off long before the adjoint's end of the list); losses
    and parameters of the persistent batched path equal the plain path's."""
    from rmesh_b200.camera import orbit_cameras

    cams = orbit_cameras(2, seed=21, radius=(2.8, 3.2), resolutions=((48, 48),))
    rng = np.random.default_rng(22)
    gts = [rng.uniform(0, 1, (48, 48, 3)).astype(np.float32) for _ in cams]
    out = {}
    for mode in ("plain", "batched"):
        r = make_renderer(c2_scene, cams[0], sh=True)
        losses = [r.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1, mode=mode, lr_sh=2.5e-3) for _ in range(2)]
        out[mode] = (np.array(losses), r.get_params(), r.info().n_pairs_last)
        r.close()
    assert out["batched"][2] / (2 * 16) > 2048  # mean tile list of more than 2,048 tets
    np.testing.assert_allclose(out["batched"][0], out["plain"][0], rtol=1e-4)
    for k in out["plain"][1]:
        assert rel_l2(out["batched"][1][k], out["plain"][1][k]) <= 1e-3, k


@pytest.mark.parametrize("jitter", [0.1, 0.0])
def test_grid_scene_parity(oracle32, jitter):
    """The reference's regular-grid mesh (test_util.rs:231-324; 8^3 vertices,
    5 tets per cell).  With jitter 0 the faces are exactly coplanar across
    cells and the axis-aligned camera's rays run exactly parallel to faces
    (the |n.d| < 1e-20 rule) and through shared edges.  Images within 1e-4,
    tile counts and sorted (tile, tet) lists bit-exact, gradients within 1e-3
    relative L2, from an axis-aligned and an oblique camera."""
    from rmesh_b200.camera import make_camera
    from rmesh_b200.scenes import grid_scene

    sc = grid_scene(8, np.random.default_rng(5), jitter=jitter)
    for eye in ((0.5, -1.6, 0.5), (1.9, -1.2, 1.4)):
        cam = make_camera(eye, (0.5, 0.5, 0.5), 50.0, 96, 96)
        r = make_renderer(sc, cam)
        img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
        ref = oracle32.forward_tiled(sc, cam)
        assert ref["P"] > 0
        np.testing.assert_array_equal(r.debug_tiles_touched(), np.where(ref["visible"] > 0, ref["tiles_touched"], 0))
        tiles, tets = r.debug_pairs()
        np.testing.assert_array_equal(tiles, ref["key_hi"])
        np.testing.assert_array_equal(tets, ref["vals"])
        assert np.abs(img - ref["image"]).max() <= 1e-4
        gt = np.random.default_rng(6).uniform(0, 1, (96, 96, 3)).astype(np.float32)
        _, dl = oracle32.loss(ref["image"], gt, 1)
        g = r.backward(dl)
        go = oracle32.backward(sc, cam, dl, ref)
        for k in go:
            assert rel_l2(g[k], go[k]) <= 1e-3, (eye, k)
        r.close()


@pytest.mark.parametrize("eye,target", [((3.0, 1.5, 0.0), (0.0, 1.5, 0.0)),     # tet at the frame's edge
                                        ((50.0, 0.0, 0.0), (0.0, 0.0, 0.0)),    # sub-pixel tet
                                        ((3.0, 0.0, 0.0), (10.0, 0.0, 0.0)),    # tet behind the camera
                                        ((3.0, 0.0, 0.0), (0.0, 0.0, 0.0))])    # centred
def test_known_tet_cross_renderer_cameras(oracle32, eye, target):
    """The camera setups of cross_renderer_test.rs:766-981 (64x64, 90 degrees)
    on the known tet: the CUDA image within 1e-4 of the oracle's, tile counts
    and (tile, tet) lists bit-exact."""
    from conftest import known_tet_scene

    from rmesh_b200.camera import make_camera

    sc = known_tet_scene()
    cam = make_camera(eye, target, 90.0, 64, 64)
    r = make_renderer(sc, cam)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(sc, cam)
    assert np.abs(img - ref["image"]).max() <= 1e-4
    np.testing.assert_array_equal(r.debug_tiles_touched(), np.where(ref["visible"] > 0, ref["tiles_touched"], 0))
    tiles, tets = r.debug_pairs()
    np.testing.assert_array_equal(tiles, ref["key_hi"])
    np.testing.assert_array_equal(tets, ref["vals"])
    r.close()


def _max_batch_items(sc, cam, ref, ts):
    """Largest number of covered (pixel, tet) items in one 32-tet batch of a
    tile's sorted list: pixel centres inside each listed tet's projected
    silhouette (convex hull of its four projected vertices), batches taken
    from the front of the list as the forward pass takes them."""
    from scipy.spatial import ConvexHull

    vp = np.asarray(cam.vp, np.float64).reshape(4, 4).T  # column-major
    v = np.asarray(sc["vertices"], np.float64).reshape(-1, 3)
    clip = np.c_[v, np.ones(len(v))] @ vp.T
    xy = clip[:, :2] / clip[:, 3:4]
    px = np.c_[(xy[:, 0] + 1) * 0.5 * cam.width, (1 - xy[:, 1]) * 0.5 * cam.height]
    idx = np.asarray(sc["indices"]).reshape(-1, 4)
    tiles_x = (cam.width + ts - 1) // ts
    real = ref["key_hi"] != 0xFFFFFFFF
    keys, vals = ref["key_hi"][real], ref["vals"][real]
    starts = np.r_[0, np.nonzero(np.diff(keys))[0] + 1, len(keys)]
    best = 0
    for a, b in zip(starts[:-1], starts[1:]):
        ty, tx = divmod(int(keys[a]), tiles_x)
        ys, xs = np.mgrid[ty * ts:(ty + 1) * ts, tx * ts:(tx + 1) * ts]
        centres = np.c_[xs.ravel() + 0.5, ys.ravel() + 0.5]
        counts = []
        for tet in vals[a:b]:
            q = px[idx[tet]]
            try:
                poly = q[ConvexHull(q).vertices]  # counter-clockwise
            except Exception:  # degenerate silhouette
                counts.append(0)
                continue
            inside = np.ones(len(centres), bool)
            for i in range(len(poly)):
                p0, p1 = poly[i], poly[(i + 1) % len(poly)]
                inside &= (p1[0] - p0[0]) * (centres[:, 1] - p0[1]) - (p1[1] - p0[1]) * (centres[:, 0] - p0[0]) >= 0
            counts.append(int(inside.sum()))
        counts = np.array(counts)[::-1]  # front to back
        for s0 in range(0, len(counts), 32):
            best = max(best, int(counts[s0:s0 + 32].sum()))
    return best


@pytest.mark.parametrize("ts", [8, 12, 16])
def test_large_tets_many_sub_batches(oracle32, ts):
    """60 points -> 287 tets, most covering more than a tile at 128x96: a
    tile's 32-tet batch then holds more covered pixels than the kernel's
    per-sub-batch item capacity (512; 800 for 12-pixel tiles), so batches
    split into sub-batches, whose item maps are written in the previous
    sub-batch's tail.  Forward image, tile
    lists, adjoint gradients, error statistics and a batched / graph-mode
    training step against the oracle."""
    from oracle import OracleTrainer
    from rmesh_b200.camera import make_camera
    from rmesh_b200.scenes import make_scene, uniform_cloud

    rng = np.random.default_rng(31)
    sc = make_scene(uniform_cloud(60, rng), rng)
    sc["densities"] = (sc["densities"] * 0.1).astype(np.float32)  # few pixels saturate
    cam = make_camera((2.2, -1.6, 1.0), (0.0, 0.0, 0.0), 60.0, 128, 96)

    r = make_renderer(sc, cam, tile_size=ts)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    ref = oracle32.forward_tiled(sc, cam, tile_size=ts)
    # some batches exceed the kernel's sub-batch capacity (953, 1,660 and 2,497
    # items at tiles of 8, 12 and 16)
    assert _max_batch_items(sc, cam, ref, ts) > (800 if ts == 12 else 512)
    tiles, tets = r.debug_pairs()
    np.testing.assert_array_equal(tiles, ref["key_hi"])
    np.testing.assert_array_equal(tets, ref["vals"])
    assert np.abs(img - ref["image"]).max() <= 1e-4

    gt = np.random.default_rng(32).uniform(0, 1, (96, 128, 3)).astype(np.float32)
    _, dl = oracle32.loss(ref["image"], gt, 1)
    g = r.backward(dl)
    go = oracle32.backward(sc, cam, dl, ref, tile_size=ts)
    for k in go:
        assert rel_l2(g[k], go[k]) <= 1e-3, k

    r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    n = cam.width * cam.height
    pe = np.random.default_rng(33).uniform(0, 1, n).astype(np.float32)
    se = np.random.default_rng(34).uniform(0, 1, n).astype(np.float32)
    err, cnt = r.forward_error(pe, se)
    e_ref, c_ref = oracle32.error_stats(sc, cam, ref, pe, se, tile_size=ts)
    for k in (0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15):
        assert rel_l2(err[:, k], e_ref[:, k]) <= 1e-4, k
    assert np.abs(cnt[:, 0] - c_ref[:, 0]).sum() <= max(2, c_ref[:, 0].sum() // 10000)
    r.close()

    cams = [cam, make_camera((-1.8, -2.0, 0.6), (0.0, 0.0, 0.0), 60.0, 128, 96)]
    gts = [gt, np.random.default_rng(35).uniform(0, 1, (96, 128, 3)).astype(np.float32)]
    for mode in ("batched", "graph"):
        r = make_renderer(sc, cam, tile_size=ts)
        tr = OracleTrainer(sc, tile_size=ts)
        for step in range(2):
            losses = r.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1, mode=mode)
            want = tr.train_step_views(cams, gts, 1e-4, 1e-2, 1e-3, 1)
            np.testing.assert_allclose(losses, want, rtol=1e-4, err_msg=f"{mode} step {step}")
        p = r.get_params()
        for k in ("vertices", "densities", "color_grads"):
            assert rel_l2(p[k], tr.scene[k]) <= 1e-3, (mode, k)
        r.close()
