"""ctypes binding of ``librmesh_b200.so`` (the C ABI in ``include/rmesh_b200.h``).

The shared library is built in-tree by ``rmesh_b200/build.py`` (nvcc, sm_100a).
There is no fallback: if the library is missing or cannot be loaded, importing
the renderer raises, so the CUDA path is always the one that runs.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# RMESH_B200_LIB selects another build of the same ABI (e.g. a profiling build)
LIB_PATH = os.environ.get("RMESH_B200_LIB") or os.path.join(_HERE, "lib", "librmesh_b200.so")

RMESH_OK = 0
RMESH_ERR_INVALID_ARG = 1
RMESH_ERR_CUDA = 2
RMESH_ERR_OOM = 3
RMESH_ERR_PAIR_OVERFLOW = 4
RMESH_ERR_TIMEOUT = 5
RMESH_ERR_STATE = 6
RMESH_ERR_NO_DEVICE = 7
RMESH_ERR_TOO_LARGE = 8
RMESH_STATIC_MAX_TETS = 1 << 24

MODE_PLAIN, MODE_BATCHED, MODE_GRAPH = 0, 1, 2
N_STAGES = 9
STAGE_NAMES = ("records", "project", "tet_sort", "emit", "pair_sort", "ranges", "composite", "adam", "sh_adjoint")

# every symbol declared in include/rmesh_b200.h
EXPORTED = (
    "rmesh_create", "rmesh_destroy", "rmesh_last_error", "rmesh_abi_version", "rmesh_set_stream",
    "rmesh_set_min_t", "rmesh_set_tile_size", "rmesh_update_params", "rmesh_get_params", "rmesh_get_info",
    "rmesh_forward_tiled", "rmesh_forward_views", "rmesh_backward",
    "rmesh_adam_state_size", "rmesh_get_adam_state", "rmesh_set_adam_state", "rmesh_train_step", "rmesh_train_step_views",
    "rmesh_debug_tiles_touched", "rmesh_debug_pairs", "rmesh_debug_ranges", "rmesh_set_profiling",
    "rmesh_stage_times", "rmesh_accumulate_views", "rmesh_grad_slots", "rmesh_apply_adam",
    "rmesh_count_tiles_static", "rmesh_update_sh", "rmesh_get_sh", "rmesh_get_sh_grad", "rmesh_set_lr_sh",
    "rmesh_decode_scene", "rmesh_forward_error", "rmesh_set_aux_data", "rmesh_get_aux_data",
    "rmesh_debug_timeouts", "rmesh_autotune_tile_size", "rmesh_backward_aux", "rmesh_set_tile_config",
    "rmesh_set_resolution_tile_config", "rmesh_get_tile_config", "rmesh_autotune",
)

COUNTERS_BYTES = 792  # sizeof(rm::Counters), read back once per training run


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int64), ("n_tets", ctypes.c_int64),
        ("vertices", ctypes.c_void_p), ("indices", ctypes.c_void_p), ("base_colors", ctypes.c_void_p),
        ("densities", ctypes.c_void_p), ("color_grads", ctypes.c_void_p), ("circumdata", ctypes.c_void_p),
        ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("aux_dim", ctypes.c_int32),
        ("tile_size", ctypes.c_int32), ("device", ctypes.c_int32), ("sh_degree", ctypes.c_int32),
        ("sh_coeffs", ctypes.c_void_p), ("reserved", ctypes.c_int32 * 2),
    ]


class PackedScene(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_uint64), ("n_tets", ctypes.c_uint64), ("sh_degree", ctypes.c_uint32),
        ("k_components", ctypes.c_uint32), ("vertices", ctypes.c_void_p), ("indices", ctypes.c_void_p),
        ("log_densities", ctypes.c_void_p), ("sh_mean", ctypes.c_void_p), ("sh_basis", ctypes.c_void_p),
        ("sh_weights", ctypes.c_void_p), ("color_grads", ctypes.c_void_p),
    ]


class Camera(ctypes.Structure):
    _fields_ = [
        ("cam_pos", ctypes.c_float * 3), ("vp", ctypes.c_float * 16), ("c2w_intrinsics", ctypes.c_float * 16),
        ("width", ctypes.c_int32), ("height", ctypes.c_int32),
    ]


class TrainOpts(ctypes.Structure):
    _fields_ = [
        ("lr_verts", ctypes.c_float), ("lr_dens", ctypes.c_float), ("lr_grads", ctypes.c_float),
        ("lr_base", ctypes.c_float), ("loss_type", ctypes.c_int32), ("mode", ctypes.c_int32),
        ("lr_sh", ctypes.c_float), ("reserved", ctypes.c_int32),
    ]


class TuneEntry(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("tile_size", ctypes.c_int32),
                ("threads", ctypes.c_int32), ("ms", ctypes.c_float)]


class Info(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int64), ("n_tets", ctypes.c_int64),
        ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("tile_size", ctypes.c_int32),
        ("n_views_last", ctypes.c_int32), ("step", ctypes.c_uint32), ("last_error_bits", ctypes.c_uint32),
        ("n_visible_last", ctypes.c_uint64), ("n_pairs_last", ctypes.c_uint64),
        ("pair_capacity", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
    ]


_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises ``OSError`` when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m rmesh_b200.build` "
                      "(nvcc, -gencode arch=compute_100a,code=sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, f32, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_float, ctypes.c_uint64
    P = ctypes.POINTER
    sig = {
        "rmesh_create": ([P(SceneDesc), P(vp)], ctypes.c_int),
        "rmesh_destroy": ([vp], ctypes.c_int),
        "rmesh_last_error": ([vp], ctypes.c_char_p),
        "rmesh_abi_version": ([], ctypes.c_int),
        "rmesh_set_stream": ([vp, vp], ctypes.c_int),
        "rmesh_set_min_t": ([vp, f32], ctypes.c_int),
        "rmesh_set_tile_size": ([vp, i32], ctypes.c_int),
        "rmesh_update_params": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_get_params": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_get_info": ([vp, P(Info)], ctypes.c_int),
        "rmesh_forward_tiled": ([vp, P(Camera), vp, vp], ctypes.c_int),
        "rmesh_forward_views": ([vp, P(Camera), i32, vp, vp], ctypes.c_int),
        "rmesh_adam_state_size": ([vp, P(ctypes.c_uint64)], ctypes.c_int),
        "rmesh_get_adam_state": ([vp, vp, P(ctypes.c_uint32)], ctypes.c_int),
        "rmesh_set_adam_state": ([vp, vp, ctypes.c_uint32], ctypes.c_int),
        "rmesh_backward": ([vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_backward_aux": ([vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_train_step": ([vp, P(Camera), vp, f32, f32, f32, i32, vp], ctypes.c_int),
        "rmesh_train_step_views": ([vp, P(Camera), i32, vp, P(TrainOpts), vp], ctypes.c_int),
        "rmesh_debug_tiles_touched": ([vp, vp], ctypes.c_int),
        "rmesh_debug_pairs": ([vp, vp, vp, u64, P(u64)], ctypes.c_int),
        "rmesh_debug_ranges": ([vp, vp, u64], ctypes.c_int),
        "rmesh_set_profiling": ([vp, i32], ctypes.c_int),
        "rmesh_stage_times": ([vp, vp, vp], ctypes.c_int),
        "rmesh_accumulate_views": ([vp, P(Camera), i32, vp, P(TrainOpts), vp], ctypes.c_int),
        "rmesh_grad_slots": ([vp, P(vp), P(u64)], ctypes.c_int),
        "rmesh_apply_adam": ([vp, P(TrainOpts)], ctypes.c_int),
        "rmesh_count_tiles_static": ([vp, u64, vp, vp, u64, P(Camera), i32, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_update_sh": ([vp, vp], ctypes.c_int),
        "rmesh_get_sh": ([vp, vp], ctypes.c_int),
        "rmesh_get_sh_grad": ([vp, vp], ctypes.c_int),
        "rmesh_set_lr_sh": ([vp, f32], ctypes.c_int),
        "rmesh_decode_scene": ([P(PackedScene), vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_forward_error": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "rmesh_set_aux_data": ([vp, vp], ctypes.c_int),
        "rmesh_get_aux_data": ([vp, vp], ctypes.c_int),
        "rmesh_debug_timeouts": ([vp], ctypes.c_int),
        "rmesh_autotune_tile_size": ([vp, P(Camera), i32, vp, P(TrainOpts), P(i32), vp], ctypes.c_int),
        "rmesh_set_tile_config": ([vp, i32, i32], ctypes.c_int),
        "rmesh_set_resolution_tile_config": ([vp, i32, i32, i32, i32], ctypes.c_int),
        "rmesh_get_tile_config": ([vp, i32, i32, P(i32), P(i32)], ctypes.c_int),
        "rmesh_autotune": ([vp, P(Camera), i32, vp, P(TrainOpts), i32, P(TuneEntry), i32, P(i32)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib
