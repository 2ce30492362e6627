"""The C-ABI library without a GPU: it loads, exports every declared symbol, its
structs match the header, and argument errors come back as status codes."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rmesh_b200.h")


def declared_symbols():
    with open(HEADER) as f:
        src = f.read()
    return sorted(set(re.findall(r"RMESH_API\s+[\w\s\*]+?\b(rmesh_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from rmesh_b200 import _lib

    lib = _lib.load()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTED) == decl
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(rmesh_\w+)\b", out))
    assert exported == set(decl)


def test_abi_version():
    from rmesh_b200 import _lib

    assert _lib.load().rmesh_abi_version() == 2


def test_struct_layouts_match_header(tmp_path):
    """Compile the header with gcc and compare sizes/offsets with the ctypes mirror."""
    from rmesh_b200 import _lib

    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "rmesh_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(RmeshSceneDesc), sizeof(RmeshCamera), sizeof(RmeshTrainOpts),
         sizeof(RmeshInfo), offsetof(RmeshSceneDesc, width));
  printf("%zu %zu %zu\n", offsetof(RmeshCamera, width), offsetof(RmeshInfo, n_visible_last),
         offsetof(RmeshTrainOpts, mode));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    a, b = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    sizes = [int(x) for x in a.split()]
    offs = [int(x) for x in b.split()]
    assert sizes == [ctypes.sizeof(_lib.SceneDesc), ctypes.sizeof(_lib.Camera), ctypes.sizeof(_lib.TrainOpts),
                     ctypes.sizeof(_lib.Info), _lib.SceneDesc.width.offset]
    assert offs == [_lib.Camera.width.offset, _lib.Info.n_visible_last.offset, _lib.TrainOpts.mode.offset]


def test_invalid_arguments_return_status():
    from rmesh_b200 import _lib

    lib = _lib.load()
    ctx = ctypes.c_void_p()
    assert lib.rmesh_create(None, ctypes.byref(ctx)) == _lib.RMESH_ERR_INVALID_ARG
    d = _lib.SceneDesc()  # zero sizes, null pointers
    assert lib.rmesh_create(ctypes.byref(d), ctypes.byref(ctx)) == _lib.RMESH_ERR_INVALID_ARG
    assert lib.rmesh_set_min_t(None, 0.5) == _lib.RMESH_ERR_INVALID_ARG
    assert lib.rmesh_destroy(None) == _lib.RMESH_OK
    assert lib.rmesh_last_error(None) == b"null context"


def _cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_available(), reason="checks the no-device path")
def test_create_without_device_fails_loudly():
    import numpy as np

    from rmesh_b200 import RMeshError, RMeshRenderer
    from conftest import known_tet_scene

    sc = known_tet_scene()
    with pytest.raises(RMeshError) as e:
        RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 64, 64)
    assert e.value.code == 7  # RMESH_ERR_NO_DEVICE: no silent CPU fallback
    assert np.isfinite(sc["vertices"]).all()


def test_renderer_validates_before_device_use():
    import numpy as np

    from rmesh_b200 import RMeshRenderer
    from conftest import known_tet_scene

    sc = known_tet_scene()
    with pytest.raises(ValueError):
        RMeshRenderer(sc["vertices"][:-1], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 64, 64)
    with pytest.raises(ValueError):
        RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"][:2], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 64, 64)
    with pytest.raises(TypeError):
        RMeshRenderer(sc["vertices"].astype(np.complex64), sc["indices"], sc["base_colors"], sc["densities"],
                      sc["color_grads"], sc["circumdata"], 64, 64)
    with pytest.raises(ValueError):
        RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                      sc["circumdata"], 64, 64, aux_dim=65)


def test_library_is_built_for_sm100a():
    """The in-tree build targets sm_100a only (no PTX for other architectures)."""
    from rmesh_b200 import build

    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "use_fast_math" not in flags
