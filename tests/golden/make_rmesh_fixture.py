"""Writes tests/golden/small_deg{1,2,3}.rmesh with the reference's own .rmesh writer.

Run from the repository root with the reference checkout available:
``python tests/golden/make_rmesh_fixture.py /path/to/rmeshvk``.

The writer is ``_process_ply_to_rmesh_buffer`` of the reference's convert.py
(convert.py:213-290): it takes a PLY read by ``tinyplypy.read_ply``, PCA-
compresses the SH coefficients (k = 12), log-encodes densities to u8 and
stores colour gradients as f16.  Its two third-party imports (tinyplypy,
pyquaternion) are not installed here; they are replaced by stand-ins that hand
the writer an in-memory PLY dictionary built from a seeded synthetic scene.
Each fixture also keeps the writer's inputs and its PCA factors
(small_deg<d>_inputs.npz: geometry, densities, colour gradients and the PCA
factors) so the tests can check the decoded scene against what went into the
file.  Degree 0 is not written: the writer's fixed k = 12 PCA components
exceed degree 0's 3 coefficients per tet, and the header it writes then
disagrees with the basis it stores.
"""
import gzip
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def synthetic_ply(seed=21, points=120, degree=3):
    sys.path.insert(0, ROOT)
    from rmesh_b200.scenes import delaunay_tets, uniform_cloud

    rng = np.random.default_rng(seed)
    pts = uniform_cloud(points, rng, -0.8, 0.8).astype(np.float32)
    tets = delaunay_tets(pts).astype(np.int32).reshape(-1, 4)
    m = tets.shape[0]
    s = np.exp(rng.normal(0.0, 1.0, m)).astype(np.float32)
    s[:5] = 1e-4  # below the writer's 1e-3 cut: these tets are dropped from the file
    nc = (degree + 1) ** 2
    tet = {"indices": tets, "s": s}
    for a, name in enumerate(("grd_x", "grd_y", "grd_z")):
        tet[name] = rng.normal(0.0, 0.1, m).astype(np.float32)
    sh = rng.normal(0.0, 0.5, (m, nc, 3)).astype(np.float32)
    for i in range(nc):
        for c, ch in enumerate("rgb"):
            tet[f"sh_{i}_{ch}"] = sh[:, i, c]
    vert = {"x": pts[:, 0], "y": pts[:, 1], "z": pts[:, 2]}
    return {"vertex": vert, "tetrahedron": tet}


def main(reference_root, degree=3):
    ply = synthetic_ply()
    stub = types.ModuleType("tinyplypy")
    stub.read_ply = lambda path: ply
    quat = types.ModuleType("pyquaternion")
    quat.Quaternion = object
    sys.modules["tinyplypy"] = stub
    sys.modules["pyquaternion"] = quat
    sys.path.insert(0, reference_root)
    import convert  # the reference's writer

    cam = np.array([0.5, -2.5, 0.8, 0.0, 0.0, 0.0, 1.0, 0.0], np.float32)
    buf, mask = convert._process_ply_to_rmesh_buffer("in-memory.ply", cam, degree)
    raw = buf.getvalue()
    with open(os.path.join(HERE, f"small_deg{degree}.rmesh"), "wb") as f:
        f.write(gzip.compress(raw, compresslevel=9, mtime=0))
    tet = ply["tetrahedron"]
    keep = ~mask
    nc = (degree + 1) ** 2
    sh = np.stack([np.stack([tet[f"sh_{i}_{ch}"] for ch in "rgb"], axis=1) for i in range(nc)], axis=1)
    sh = np.transpose(sh, (0, 2, 1))[keep]  # [M, 3, nc] of the written degree, as the writer lays it out
    w16, b16, m16 = convert.compress_matrix(sh, k=12)  # the factors the writer stored
    v = ply["vertex"]
    np.savez_compressed(os.path.join(HERE, f"small_deg{degree}_inputs.npz"),
                        vertices=np.stack([v["x"], v["y"], v["z"]], axis=1).astype(np.float32),
                        indices=tet["indices"][keep].astype(np.uint32), densities=tet["s"][keep],
                        color_grads=np.stack([tet["grd_x"], tet["grd_y"], tet["grd_z"]], axis=1)[keep],
                        pca_weights=w16, pca_basis=b16, pca_mean=m16, start_pose=cam)
    print(f"degree {degree}: wrote", len(raw), "bytes raw;", int(keep.sum()), "tets kept of", keep.size)


if __name__ == "__main__":
    for d in (1, 2, 3):
        main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.sep, "root", "reference"), d)
