""".rmesh scene files: the oracle's decode pinned to the reference's writer,
the host section parser, and the device decode (bit-exact vs the oracle).

tests/golden/small_deg{1,2,3}.rmesh were written by the reference's own writer
(convert.py:213-290, see tests/golden/make_rmesh_fixture.py) from a seeded
615-tet scene at SH degrees 1, 2 and 3; small_deg<d>_inputs.npz hold what went
into them.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT, c1_camera

DEGREES = (1, 2, 3)


def _fix(deg):
    return os.path.join(ROOT, "tests", "golden", f"small_deg{deg}.rmesh")


def _inp(deg):
    return os.path.join(ROOT, "tests", "golden", f"small_deg{deg}_inputs.npz")


FIX = _fix(3)


def _raw(deg=3):
    from rmesh_b200.rmesh_file import read_rmesh_bytes

    return read_rmesh_bytes(_fix(deg))


@pytest.mark.parametrize("deg", DEGREES)
def test_oracle_decode_matches_reference_writer(oracle32, deg):
    """Decoding (crates/rmesh-data/src/lib.rs:247-393) returns what the writer
    stored: exact geometry, densities within the u8 log code's step
    (exp(1/20) = 5.1 %), colour gradients within f16, SH equal to the PCA
    reconstruction of the writer's factors, circumspheres as computed here."""
    from rmesh_b200.scenes import circumspheres

    d = oracle32.rmesh_decode(_raw(deg))
    g = np.load(_inp(deg))
    assert d["sh_degree"] == deg
    assert d["sh_coeffs"].size == 615 * 3 * (deg + 1) ** 2
    np.testing.assert_array_equal(d["vertices"], g["vertices"].ravel())
    np.testing.assert_array_equal(d["indices"], g["indices"].ravel())
    np.testing.assert_array_equal(d["start_pose"], g["start_pose"][:7])
    rel = d["densities"] / g["densities"]
    assert np.all(rel <= 1.0 + 1e-6) and np.all(rel > np.exp(-1.0 / 20.0) - 1e-6)  # u8 code truncates
    np.testing.assert_array_equal(d["color_grads"], g["color_grads"].astype(np.float16).astype(np.float32).ravel())
    rec = g["pca_mean"].astype(np.float64)[None, :] + g["pca_weights"].astype(np.float64) @ g["pca_basis"].astype(
        np.float64)
    np.testing.assert_allclose(d["sh_coeffs"], rec.ravel(), atol=2e-3)
    np.testing.assert_array_equal(d["circumdata"], circumspheres(d["vertices"], d["indices"]))


@pytest.mark.parametrize("deg", DEGREES)
def test_host_sections(oracle32, deg):
    from rmesh_b200.rmesh_file import parse_rmesh_sections

    raw = _raw(deg)
    sec = parse_rmesh_sections(raw)
    d = oracle32.rmesh_decode(raw)
    assert (sec["n_vertices"], sec["n_tets"], sec["sh_degree"], sec["k_components"]) == (120, 615, deg, 12)
    np.testing.assert_array_equal(sec["vertices"], d["vertices"])
    np.testing.assert_array_equal(sec["indices"], d["indices"])
    np.testing.assert_array_equal(sec["color_grads_f16"].view(np.float16).astype(np.float32), d["color_grads"])
    assert sec["sh_weights"].size == 615 * 12 and sec["sh_basis"].size == 12 * 3 * (deg + 1) ** 2


def test_truncated_and_tagged_files(oracle32):
    from rmesh_b200.rmesh_file import parse_rmesh_sections

    raw = _raw()
    for cut in (20, 48 + 100, len(raw) - 3 * 615 * 2 - 200):
        with pytest.raises(ValueError):
            parse_rmesh_sections(raw[:cut])
    # a tagged section where the gradients would start: gradients read as zeros
    # (lib.rs:305-310)
    sec = parse_rmesh_sections(raw)
    goff = len(raw) - 3 * 615 * 2
    tagged = raw[:goff] + np.array([0x524D5458], np.uint32).tobytes() + bytes(64)
    assert parse_rmesh_sections(tagged)["color_grads_f16"] is None
    assert np.all(oracle32.rmesh_decode(tagged)["color_grads"] == 0.0)
    # a short gradient section is zero-padded (lib.rs:313-321)
    short = raw[:goff + 100]
    g = parse_rmesh_sections(short)["color_grads_f16"]
    assert g.size == 3 * 615 and np.all(g[50:] == 0) and np.array_equal(g[:50], sec["color_grads_f16"][:50])


@pytest.mark.gpu
@pytest.mark.parametrize("deg", DEGREES)
def test_device_decode_matches_oracle(oracle32, deg):
    from rmesh_b200.rmesh_file import load_rmesh

    d = oracle32.rmesh_decode(_raw(deg))
    s = load_rmesh(_fix(deg))
    for k in ("vertices", "densities", "color_grads", "circumdata", "sh_coeffs"):
        np.testing.assert_array_equal(s[k].cpu().numpy(), d[k], err_msg=k)
    np.testing.assert_array_equal(s["indices"].cpu().numpy().view(np.uint32), d["indices"])


@pytest.mark.gpu
@pytest.mark.parametrize("deg", DEGREES)
def test_loaded_scene_renders_like_oracle(oracle32, deg):
    """A renderer built straight from the device tensors of load_rmesh."""
    from rmesh_b200 import RMeshRenderer
    from rmesh_b200.rmesh_file import load_rmesh

    s = load_rmesh(_fix(deg))
    cam = c1_camera(160, 128)
    r = RMeshRenderer(s["vertices"], s["indices"], s["base_colors"], s["densities"], s["color_grads"],
                      s["circumdata"], cam.width, cam.height, sh_coeffs=s["sh_coeffs"], sh_degree=s["sh_degree"])
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    d = oracle32.rmesh_decode(_raw(deg))
    scene = {k: d[k] for k in ("vertices", "indices", "densities", "color_grads", "circumdata")}
    scene["base_colors"] = s["base_colors"].cpu().numpy()
    ref = oracle32.forward_tiled(scene, cam, sh=oracle32.sh_values(d["sh_coeffs"]), sh_degree=deg)
    assert ref["image"][..., 3].max() > 0.1
    assert np.abs(img - ref["image"]).max() <= 1e-4
