"""Generates the golden fixtures in this folder (run from the repository root:
``python tests/golden/make_golden.py``).

They freeze, on the reference's own test fixtures, the outputs the parity tests
rely on, so that a change to the CPU oracle or to the numpy restatement of the
reference's CPU renderer shows up as a golden mismatch:

* known_tet.npz   -- oracle (float32), known regular tet (kernel_tests.rs:1516-1545)
                     seen from (0,-2,0.5), 64x64, tile 12: image, tiles_touched,
                     sorted tile ids / tet ids, tile ranges
* two_tet.npz     -- oracle (float64), two-tet scene (kernel_tests.rs:61-88) from
                     (3,0.4,1): image, L2-vs-gray loss, analytic gradients, and
                     central finite differences (eps 1e-3) of the density gradients
* four_tet_cpu.npz -- numpy restatement of the reference CPU renderer
                     (common/mod.rs:240-351), four-tet scene from (2,2,2)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

from conftest import known_tet_scene, two_tet_scene  # noqa: E402
from oracle import Oracle  # noqa: E402
from ref_cpu_renderer import cpu_render_scene  # noqa: E402
from rmesh_b200.camera import make_camera  # noqa: E402
from test_oracle import four_tet_scene  # noqa: E402


def main():
    o32, o64 = Oracle("f32"), Oracle("f64")
    cam = make_camera((0.0, -2.0, 0.5), (0, 0, 0), 90.0, 64, 64)
    f = o32.forward_tiled(known_tet_scene(), cam)
    np.savez_compressed(os.path.join(HERE, "known_tet.npz"), image=f["image"], tiles_touched=f["tiles_touched"],
                        tiles=f["key_hi"], tets=f["vals"], ranges=f["ranges"])

    sc = {k: (np.asarray(v, np.float64) if v.dtype.kind == "f" else v) for k, v in two_tet_scene().items()}
    cam2 = make_camera((3.0, 0.4, 1.0), (0.5, 0.4, 0.0), 90.0, 64, 64)
    gt = np.full((64, 64, 3), 0.5)
    f2 = o64.forward_tiled(sc, cam2)
    loss, dl = o64.loss(f2["image"], gt, 1)
    g = o64.backward(sc, cam2, dl, f2)
    fd = []
    for i in range(sc["densities"].size):
        vals = []
        for s in (1, -1):
            sp = {k: v.copy() for k, v in sc.items()}
            sp["densities"][i] += s * 1e-3
            vals.append(o64.loss(o64.forward_tiled(sp, cam2)["image"], gt, 1)[0])
        fd.append((vals[0] - vals[1]) / 2e-3)
    np.savez_compressed(os.path.join(HERE, "two_tet.npz"), image=f2["image"], loss=loss, fd_densities=np.array(fd),
                        **g)

    sc4 = four_tet_scene()
    cam4 = make_camera((2.0, 2.0, 2.0), (0, 0, 0), 90.0, 64, 64)
    np.savez_compressed(os.path.join(HERE, "four_tet_cpu.npz"), image=cpu_render_scene(sc4, cam4))


if __name__ == "__main__":
    main()
