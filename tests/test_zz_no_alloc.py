"""rmesh_count_tiles_static: the allocation-free tile count, through the C ABI.

Its per-tet tile counts must equal, bit for bit, the tiles_touched that the
context path reports after a single-view forward (rmesh_debug_tiles_touched),
and its visible list must be exactly the tets with a non-zero count, in
ascending order.  Two calls run back to back on the same output buffers, so the
second one also checks that each call re-clears the shared scratch.  The file
name sorts last so the test also runs after every other GPU test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import c1_camera, make_renderer


def _cam_struct(cam):
    from rmesh_b200.renderer import _camera_struct

    return _camera_struct(cam.cam_pos, cam.vp, cam.c2w_intrinsics, cam.width, cam.height)


def _call(lib, dev, cam, tile_size, out, stream=None):
    vert, idx, dens = dev
    tiles, visible, counts = out
    cs = _cam_struct(cam)
    return lib.rmesh_count_tiles_static(vert.data_ptr(), vert.numel() // 3, idx.data_ptr(), dens.data_ptr(),
                                        dens.numel(), ctypes.byref(cs), tile_size, tiles.data_ptr(),
                                        visible.data_ptr(), counts.data_ptr(), stream)


def test_rejects_oversize_and_missing_arguments():
    from rmesh_b200 import _lib
    from rmesh_b200.camera import make_camera

    lib = _lib.load()
    cs = _cam_struct(make_camera((0, -2, 0.5), (0, 0, 0), 60.0, 64, 64))
    big = _lib.RMESH_STATIC_MAX_TETS + 1
    assert lib.rmesh_count_tiles_static(None, 4, None, None, big, ctypes.byref(cs), 12, None, None, None,
                                        None) == _lib.RMESH_ERR_TOO_LARGE
    assert lib.rmesh_count_tiles_static(None, 4, None, None, 1, None, 12, None, None, None,
                                        None) == _lib.RMESH_ERR_INVALID_ARG
    assert lib.rmesh_count_tiles_static(None, 4, None, None, 1, ctypes.byref(cs), 12, None, None, None,
                                        None) == _lib.RMESH_ERR_INVALID_ARG


@pytest.mark.gpu
def test_static_count_matches_context_path_twice(c1_scene):
    import torch

    from rmesh_b200 import _lib
    from rmesh_b200.camera import make_camera

    lib = _lib.load()
    sc = c1_scene
    M = sc["densities"].size
    dev = (torch.from_numpy(sc["vertices"]).cuda(),
           torch.from_numpy(sc["indices"].view(np.int32)).cuda(),
           torch.from_numpy(sc["densities"]).cuda())
    # outputs belong to the caller; poison them so stale values cannot pass
    out = (torch.full((M,), -1, dtype=torch.int32, device="cuda"),
           torch.full((M,), -1, dtype=torch.int32, device="cuda"),
           torch.full((2,), -1, dtype=torch.int32, device="cuda"))
    cases = [(c1_camera(512, 512), 12), (make_camera((2.2, 1.4, -0.9), (0.1, 0, 0), 50.0, 200, 120), 16)]
    for cam, ts in cases:
        r = make_renderer(sc, cam, tile_size=ts)
        r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
        want = r.debug_tiles_touched()
        r.close()

        assert _call(lib, dev, cam, ts, out) == _lib.RMESH_OK
        torch.cuda.synchronize()
        tiles = out[0].cpu().numpy().view(np.uint32)
        visible = out[1].cpu().numpy().view(np.uint32)
        n_vis, err = (int(x) for x in out[2].cpu().numpy().view(np.uint32))
        assert err == 0
        np.testing.assert_array_equal(tiles, want)
        expect_ids = np.nonzero(want)[0].astype(np.uint32)
        assert n_vis == expect_ids.size > 0
        np.testing.assert_array_equal(visible[:n_vis], expect_ids)


@pytest.mark.gpu
def test_static_count_rejects_host_memory(c1_scene):
    import torch

    from rmesh_b200 import _lib

    lib = _lib.load()
    sc = c1_scene
    M = sc["densities"].size
    cs = _cam_struct(c1_camera(64, 64))
    host_out = np.zeros(M, np.uint32)
    counts = torch.zeros(2, dtype=torch.int32, device="cuda")
    rc = lib.rmesh_count_tiles_static(sc["vertices"].ctypes.data, sc["vertices"].size // 3,
                                      sc["indices"].ctypes.data, sc["densities"].ctypes.data, M, ctypes.byref(cs),
                                      12, host_out.ctypes.data, host_out.ctypes.data, counts.data_ptr(), None)
    assert rc == _lib.RMESH_ERR_INVALID_ARG


@pytest.mark.gpu
def test_static_count_bad_index_empty_mesh_and_no_allocation(c1_scene):
    """A tet with a vertex index past the vertex count is skipped and flagged
    (counts[1] bit 4) while every other tet keeps its count; an empty mesh
    returns counts (0, 0); and a warm call leaves the device's free memory
    unchanged (the call allocates nothing)."""
    import torch

    from rmesh_b200 import _lib

    lib = _lib.load()
    sc = c1_scene
    M = sc["densities"].size
    N = sc["vertices"].size // 3
    cam = c1_camera(256, 256)
    vert = torch.from_numpy(sc["vertices"]).cuda()
    dens = torch.from_numpy(sc["densities"]).cuda()
    good = torch.from_numpy(sc["indices"].view(np.int32)).cuda()
    out = (torch.full((M,), -1, dtype=torch.int32, device="cuda"),
           torch.full((M,), -1, dtype=torch.int32, device="cuda"),
           torch.full((2,), -1, dtype=torch.int32, device="cuda"))
    assert _call(lib, (vert, good, dens), cam, 12, out) == _lib.RMESH_OK
    torch.cuda.synchronize()
    want = out[0].cpu().numpy().view(np.uint32).copy()
    hit = int(np.nonzero(want)[0][0])  # a tile-touching tet, made invalid below

    bad_idx = sc["indices"].copy()
    bad_idx[4 * hit + 2] = N  # one past the last vertex
    bad = torch.from_numpy(bad_idx.view(np.int32)).cuda()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert _call(lib, (vert, bad, dens), cam, 12, out) == _lib.RMESH_OK
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0
    tiles = out[0].cpu().numpy().view(np.uint32)
    n_vis, err = (int(x) for x in out[2].cpu().numpy().view(np.uint32))
    assert err & 4
    assert tiles[hit] == 0
    rest = np.ones(M, bool)
    rest[hit] = False
    np.testing.assert_array_equal(tiles[rest], want[rest])
    assert n_vis == int(np.count_nonzero(want)) - 1

    # empty mesh: counts cleared to (0, 0), nothing else touched
    counts = torch.full((2,), -1, dtype=torch.int32, device="cuda")
    cs = _cam_struct(cam)
    assert lib.rmesh_count_tiles_static(None, 0, None, None, 0, ctypes.byref(cs), 12, None, None,
                                        counts.data_ptr(), None) == _lib.RMESH_OK
    torch.cuda.synchronize()
    assert counts.cpu().tolist() == [0, 0]
