"""``RMeshRenderer``: the reference binding's class, backed by the B200 C ABI.

Method names, argument meaning, dict keys and return shapes follow the PyO3
class of the reference (crates/rmesh-python/src/lib.rs):

* ``RMeshRenderer(vertices, indices, base_colors, densities, color_grads,
  circumdata, width, height, aux_dim=0)``                       lib.rs:265-277
* ``set_min_t(min_t)``                                          lib.rs:873-875
* ``forward_tiled(cam_pos, vp, c2w_intrinsics, render_aux=False)`` lib.rs:1040-1204
* ``backward(dl_d_image) -> dict``                              lib.rs:1894-2031
* ``train_step(cam_pos, vp, c2w_intrinsics, gt_image, lr_verts, lr_dens,
  lr_grads, loss_type) -> float``                               lib.rs:2405-2636
* ``update_params(...)`` / ``get_params()``                     lib.rs:2641-2686
* ``step`` / ``width`` / ``height``                             lib.rs:2688-2705

Differences, all additive: ``train_step`` returns the actual loss (the
reference returns 0.0 because its loss buffer is never written); inputs may
also be torch tensors, and CUDA tensors are passed to the device without a
host round trip; ``train_step_views`` trains on several cameras per step.
"""
from __future__ import annotations

import ctypes
import sys
from typing import Sequence

import numpy as np

from . import _lib
from .staging import StagedTargets

__all__ = ["RMeshRenderer", "RMeshError"]


class RMeshError(RuntimeError):
    """A failing C-ABI call (status code and message attached)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"rmesh_b200 error {code}: {msg}")
        self.code = code


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _as_array(x, dtype, name: str):
    """Returns (object to keep alive, pointer as int) for a flat C-contiguous array."""
    if _is_torch(x):
        import torch

        tdt = torch.float32 if dtype == np.float32 else torch.int32
        if x.dtype not in (tdt, torch.uint32 if dtype == np.uint32 else tdt):
            if dtype == np.uint32 and x.dtype in (torch.int32, torch.int64):
                x = x.to(torch.int32)
            else:
                raise TypeError(f"{name}: expected a {tdt} tensor, got {x.dtype}")
        x = x.contiguous()
        # the library reads the tensor on its own stream: finish torch's pending
        # work on it first (including the copy contiguous() may have queued)
        if x.is_cuda:
            torch.cuda.current_stream(x.device).synchronize()
        return x, x.data_ptr()
    a = np.asarray(x)
    if a.dtype != dtype:
        if dtype == np.uint32 and a.dtype.kind in "iu":
            a = a.astype(np.uint32)
        elif dtype == np.float32 and a.dtype.kind == "f":
            a = a.astype(np.float32)
        else:
            raise TypeError(f"{name}: expected {np.dtype(dtype).name}, got {a.dtype}")
    a = np.ascontiguousarray(a)
    return a, a.ctypes.data


def _camera_struct(cam_pos, vp, c2w_intrinsics, width: int, height: int) -> _lib.Camera:
    c = _lib.Camera()
    cp = np.asarray(_to_numpy(cam_pos), dtype=np.float32).ravel()
    v = np.asarray(_to_numpy(vp), dtype=np.float32).ravel()
    ci = np.asarray(_to_numpy(c2w_intrinsics), dtype=np.float32).ravel()
    if cp.size != 3 or v.size != 16 or ci.size != 16:
        raise ValueError("cam_pos must have 3 values, vp and c2w_intrinsics 16")
    c.cam_pos[:] = cp.tolist()
    c.vp[:] = v.tolist()
    c.c2w_intrinsics[:] = ci.tolist()
    c.width = int(width)
    c.height = int(height)
    return c


def _to_numpy(x):
    if _is_torch(x):
        return x.detach().cpu().numpy()
    return x


class RMeshRenderer:
    """Tiled differentiable tet-mesh volume renderer on one CUDA device."""

    def __init__(self, vertices, indices, base_colors, densities, color_grads, circumdata, width: int,
                 height: int, aux_dim: int = 0, *, tile_size: int = 12, device: int | None = None,
                 sh_coeffs=None, sh_degree: int | None = None):
        """Arguments as the reference's constructor (crates/rmesh-python/src/lib.rs:265-277).
        ``sh_coeffs`` ([M, 3, (sh_degree+1)^2] floats, no reference counterpart in
        the binding) switches the colours from ``base_colors`` to the reference
        shader's view-dependent SH colour (project_compute.wgsl:264-318)."""
        self._lib = _lib.load()
        if not 0 <= int(aux_dim) <= 64:
            raise ValueError("aux_dim must be 0..64")
        self._aux_dim = int(aux_dim)
        keep = []
        ptrs = {}
        for name, arr, dt in (("vertices", vertices, np.float32), ("indices", indices, np.uint32),
                              ("base_colors", base_colors, np.float32), ("densities", densities, np.float32),
                              ("color_grads", color_grads, np.float32), ("circumdata", circumdata, np.float32)):
            obj, p = _as_array(arr, dt, name)
            keep.append(obj)
            ptrs[name] = (obj, p)
        n_v = _numel(ptrs["vertices"][0])
        n_i = _numel(ptrs["indices"][0])
        if n_v % 3 or n_i % 4 or n_i == 0:
            raise ValueError("vertices must hold 3N floats and indices 4M (M > 0) integers")
        self._N, self._M = n_v // 3, n_i // 4
        idx_obj = ptrs["indices"][0]
        if isinstance(idx_obj, np.ndarray) and int(idx_obj.max()) >= self._N:
            raise ValueError(f"indices must be below the vertex count {self._N}")  # device arrays: checked in C
        for name, per in (("base_colors", 3), ("densities", 1), ("color_grads", 3), ("circumdata", 4)):
            if _numel(ptrs[name][0]) != per * self._M:
                raise ValueError(f"{name} must hold {per}*M = {per * self._M} values")
        self._sh_degree = -1
        self._nc = 0
        if sh_coeffs is not None:
            obj, p_sh = _as_array(sh_coeffs, np.float32, "sh_coeffs")
            n_sh = _numel(obj)
            if sh_degree is None:
                nc = n_sh // (3 * self._M)
                sh_degree = int(round(nc ** 0.5)) - 1
            if not 0 <= int(sh_degree) <= 3:
                raise ValueError("sh_degree must be 0..3")
            self._sh_degree, self._nc = int(sh_degree), (int(sh_degree) + 1) ** 2
            if n_sh != 3 * self._nc * self._M:
                raise ValueError(f"sh_coeffs must hold 3*(sh_degree+1)^2*M = {3 * self._nc * self._M} values")
            keep.append(obj)
        d = _lib.SceneDesc()
        d.n_vertices, d.n_tets = self._N, self._M
        if self._sh_degree >= 0:
            d.sh_coeffs, d.sh_degree = p_sh, self._sh_degree
        d.vertices, d.indices = ptrs["vertices"][1], ptrs["indices"][1]
        d.base_colors, d.densities = ptrs["base_colors"][1], ptrs["densities"][1]
        d.color_grads, d.circumdata = ptrs["color_grads"][1], ptrs["circumdata"][1]
        d.width, d.height, d.aux_dim, d.tile_size = int(width), int(height), self._aux_dim, int(tile_size)
        d.device = -1 if device is None else int(device)
        ctx = ctypes.c_void_p()
        rc = self._lib.rmesh_create(ctypes.byref(d), ctypes.byref(ctx))
        if rc != 0:
            raise RMeshError(rc, "rmesh_create failed (no CUDA device, bad sizes, an index not below the vertex "
                                 "count, or out of memory)")
        self._ctx = ctx
        self._width, self._height = int(width), int(height)
        self._tile_size = int(tile_size)
        torch = sys.modules.get("torch")
        if device is None and torch is not None and torch.cuda.is_available():
            device = torch.cuda.current_device()
        self._device_index = None if device is None else int(device)
        self._stream_handle = None  # set by set_stream
        self._torch_stream = None

    # ------------------------------------------------------------------ utils
    def _check(self, rc: int):
        if rc != 0:
            msg = self._lib.rmesh_last_error(self._ctx)
            raise RMeshError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.rmesh_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _cam(self, cam_pos, vp, c2w_intrinsics, width=None, height=None):
        return _camera_struct(cam_pos, vp, c2w_intrinsics, self._width if width is None else width,
                              self._height if height is None else height)

    # ---------------------------------------------------------------- getters
    @property
    def step(self) -> int:
        return int(self.info().step)

    @property
    def width(self) -> int:
        return self._width

    @property
    def height(self) -> int:
        return self._height

    @property
    def n_vertices(self) -> int:
        return self._N

    @property
    def n_tets(self) -> int:
        return self._M

    @property
    def sh_degree(self) -> int:
        """-1 when colours are base_colors, else the SH degree."""
        return self._sh_degree

    def info(self) -> _lib.Info:
        inf = _lib.Info()
        self._check(self._lib.rmesh_get_info(self._ctx, ctypes.byref(inf)))
        return inf

    # --------------------------------------------------------------- settings
    def set_min_t(self, min_t: float):
        self._check(self._lib.rmesh_set_min_t(self._ctx, float(min_t)))

    def set_tile_size(self, tile_size: int):
        self._check(self._lib.rmesh_set_tile_size(self._ctx, int(tile_size)))
        self._tile_size = int(tile_size)

    def set_tile_config(self, tile_size: int, threads: int = 0):
        """Default tile configuration: tile size 8, 12 or 16 and threads per
        tile (0: one per pixel rounded up to warps; or twice that)."""
        self._check(self._lib.rmesh_set_tile_config(self._ctx, int(tile_size), int(threads)))
        self._tile_size = int(tile_size)

    def set_resolution_tile_config(self, width: int, height: int, tile_size: int, threads: int = 0):
        """Views of width x height use this configuration (tile_size 0 removes it)."""
        self._check(self._lib.rmesh_set_resolution_tile_config(self._ctx, int(width), int(height), int(tile_size),
                                                                int(threads)))

    def tile_config(self, width: int = 0, height: int = 0):
        """(tile_size, threads per tile) a view of width x height runs with (0, 0: the default)."""
        ts, th = ctypes.c_int32(0), ctypes.c_int32(0)
        self._check(self._lib.rmesh_get_tile_config(self._ctx, int(width), int(height), ctypes.byref(ts),
                                                     ctypes.byref(th)))
        return int(ts.value), int(th.value)

    def set_stream(self, stream_handle: int):
        self._check(self._lib.rmesh_set_stream(self._ctx, ctypes.c_void_p(int(stream_handle))))
        self._stream_handle = int(stream_handle)
        self._torch_stream = None

    @property
    def device_index(self) -> int:
        """The CUDA device ordinal of this renderer."""
        if self._device_index is None:
            import torch

            self._device_index = torch.cuda.current_device()
        return self._device_index

    def torch_stream(self):
        """The renderer's CUDA stream as a torch stream.  Without an earlier
        ``set_stream`` this creates a torch stream and makes it the renderer's."""
        import torch

        if self._torch_stream is None:
            if self._stream_handle is None:
                st = torch.cuda.Stream(device=self.device_index)
                self.set_stream(st.cuda_stream)
                self._torch_stream = st
            else:
                self._torch_stream = torch.cuda.ExternalStream(self._stream_handle, device=self.device_index)
        return self._torch_stream

    # ------------------------------------------------------------- parameters
    def update_params(self, vertices, base_colors, densities, color_grads, sh_coeffs=None):
        keep = []
        if sh_coeffs is not None:
            if self._sh_degree < 0:
                raise ValueError("this renderer has no SH coefficients")
            obj, p = _as_array(sh_coeffs, np.float32, "sh_coeffs")
            if _numel(obj) != 3 * self._nc * self._M:
                raise ValueError("sh_coeffs has the wrong size")
            keep.append(obj)
            self._check(self._lib.rmesh_update_sh(self._ctx, p))
        ps = []
        for name, arr, n in (("vertices", vertices, 3 * self._N), ("base_colors", base_colors, 3 * self._M),
                             ("densities", densities, self._M), ("color_grads", color_grads, 3 * self._M)):
            if arr is None:
                ps.append(None)
                continue
            obj, p = _as_array(arr, np.float32, name)
            if _numel(obj) != n:
                raise ValueError(f"{name} must hold {n} values, got {_numel(obj)}")
            keep.append(obj)
            ps.append(p)
        self._check(self._lib.rmesh_update_params(self._ctx, *ps))

    def get_params(self) -> dict:
        out = {"vertices": np.empty(3 * self._N, np.float32), "base_colors": np.empty(3 * self._M, np.float32),
               "densities": np.empty(self._M, np.float32), "color_grads": np.empty(3 * self._M, np.float32)}
        self._check(self._lib.rmesh_get_params(self._ctx, out["vertices"].ctypes.data,
                                               out["base_colors"].ctypes.data, out["densities"].ctypes.data,
                                               out["color_grads"].ctypes.data))
        if self._sh_degree >= 0:
            out["sh_coeffs"] = np.empty(3 * self._nc * self._M, np.float32)
            self._check(self._lib.rmesh_get_sh(self._ctx, out["sh_coeffs"].ctypes.data))
        return out

    def state_dict(self) -> dict:
        """Checkpoint: parameters (as ``get_params``), the Adam moments of
        every group (one float32 array, see ``rmesh_get_adam_state``) and the
        step count.  No reference counterpart (its Adam state is private)."""
        n = ctypes.c_uint64()
        self._check(self._lib.rmesh_adam_state_size(self._ctx, ctypes.byref(n)))
        adam = np.empty(int(n.value), np.float32)
        step = ctypes.c_uint32()
        self._check(self._lib.rmesh_get_adam_state(self._ctx, adam.ctypes.data, ctypes.byref(step)))
        return {"params": self.get_params(), "adam": adam, "step": int(step.value)}

    def load_state_dict(self, state: dict):
        """Restores a ``state_dict`` of a renderer over the same mesh; training
        then continues as it would have from the saved state."""
        p = state["params"]
        self.update_params(p["vertices"], p["base_colors"], p["densities"], p["color_grads"],
                           sh_coeffs=p.get("sh_coeffs"))
        n = ctypes.c_uint64()
        self._check(self._lib.rmesh_adam_state_size(self._ctx, ctypes.byref(n)))
        adam = np.ascontiguousarray(state["adam"], dtype=np.float32)
        if adam.size != int(n.value):
            raise ValueError(f"adam state must hold {int(n.value)} floats, got {adam.size}")
        self._check(self._lib.rmesh_set_adam_state(self._ctx, adam.ctypes.data, int(state["step"])))

    def sh_grad_into(self, out):
        """Coefficient gradient of the last backward / training call into ``out``."""
        _, p = _as_array(out, np.float32, "out")
        self._check(self._lib.rmesh_get_sh_grad(self._ctx, p))
        return out

    # -------------------------------------------------------------- the path
    def set_aux_data(self, aux_data):
        """Per-tet custom aux channels [M * aux_dim] (lib.rs:892-910)."""
        if self._aux_dim == 0:
            raise ValueError("aux_dim is 0; construct with aux_dim > 0 to use custom aux channels")
        obj, p = _as_array(aux_data, np.float32, "aux_data")
        if _numel(obj) != self._M * self._aux_dim:
            raise ValueError(f"Expected {self._M * self._aux_dim} elements (tet_count={self._M} * "
                             f"aux_dim={self._aux_dim}), got {_numel(obj)}")
        self._check(self._lib.rmesh_set_aux_data(self._ctx, p))

    def get_aux_data(self) -> np.ndarray:
        if self._aux_dim == 0:
            raise ValueError("aux_dim is 0; no aux data to read")
        out = np.empty(self._M * self._aux_dim, np.float32)
        self._check(self._lib.rmesh_get_aux_data(self._ctx, out.ctypes.data))
        return out

    def forward_tiled(self, cam_pos, vp, c2w_intrinsics, render_aux: bool = False):
        """[H, W, 4] premultiplied RGBA (and [H, W, 8 + aux_dim] aux when ``render_aux``)."""
        cam = self._cam(cam_pos, vp, c2w_intrinsics)
        rgba = np.empty((self._height, self._width, 4), np.float32)
        aux = np.empty((self._height, self._width, 8 + self._aux_dim), np.float32) if render_aux else None
        self._check(self._lib.rmesh_forward_tiled(self._ctx, ctypes.byref(cam), rgba.ctypes.data,
                                                  aux.ctypes.data if render_aux else None))
        return (rgba, aux) if render_aux else rgba

    def forward_tiled_into(self, cam_pos, vp, c2w_intrinsics, out, aux_out=None):
        """Device-tensor variant: writes into ``out`` ([H,W,4] float32, host or CUDA)."""
        cam = self._cam(cam_pos, vp, c2w_intrinsics)
        _, p = _as_array(out, np.float32, "out")
        pa = None if aux_out is None else _as_array(aux_out, np.float32, "aux_out")[1]
        self._check(self._lib.rmesh_forward_tiled(self._ctx, ctypes.byref(cam), p, pa))
        return out

    def backward(self, dl_d_image, dl_d_aux=None) -> dict:
        """dict of 1-D float32 arrays d_vertices, d_densities, d_base_colors, d_color_grads
        (and d_sh_coeffs when the colours come from SH coefficients).

        With custom aux channels (``aux_dim`` > 0) the dict also holds
        ``d_aux_data`` [M * aux_dim], and ``dl_d_aux`` ([H, W, aux_dim], the loss
        gradient of the aux image's custom channels; None = zero) contributes
        to every gradient, as the reference's ``dl_d_aux`` argument
        (crates/rmesh-python/src/lib.rs:2043-2090)."""
        obj, p = _as_array(dl_d_image, np.float32, "dl_d_image")
        if _numel(obj) != 4 * self._width * self._height:
            raise ValueError("dl_d_image must be [H, W, 4]")
        out = {"d_vertices": np.empty(3 * self._N, np.float32), "d_densities": np.empty(self._M, np.float32),
               "d_base_colors": np.empty(3 * self._M, np.float32),
               "d_color_grads": np.empty(3 * self._M, np.float32)}
        if self._aux_dim > 0:
            pa = None
            if dl_d_aux is not None:
                aobj, pa = _as_array(dl_d_aux, np.float32, "dl_d_aux")
                if _numel(aobj) != self._aux_dim * self._width * self._height:
                    raise ValueError("dl_d_aux must be [H, W, aux_dim]")
            out["d_aux_data"] = np.empty(self._aux_dim * self._M, np.float32)
            self._check(self._lib.rmesh_backward_aux(self._ctx, p, pa, out["d_vertices"].ctypes.data,
                                                     out["d_densities"].ctypes.data,
                                                     out["d_base_colors"].ctypes.data,
                                                     out["d_color_grads"].ctypes.data,
                                                     out["d_aux_data"].ctypes.data))
        else:
            if dl_d_aux is not None:
                raise ValueError("dl_d_aux needs a renderer with aux_dim > 0")
            self._check(self._lib.rmesh_backward(self._ctx, p, out["d_vertices"].ctypes.data,
                                                 out["d_densities"].ctypes.data, out["d_base_colors"].ctypes.data,
                                                 out["d_color_grads"].ctypes.data))
        if self._sh_degree >= 0:
            out["d_sh_coeffs"] = self.sh_grad_into(np.empty(3 * self._nc * self._M, np.float32))
        return out

    def backward_into(self, dl_d_image, d_vertices, d_densities, d_base_colors, d_color_grads):
        """Device-tensor variant of ``backward`` writing into the given buffers."""
        _, p = _as_array(dl_d_image, np.float32, "dl_d_image")
        ptrs = [_as_array(t, np.float32, "grad")[1] if t is not None else None
                for t in (d_vertices, d_densities, d_base_colors, d_color_grads)]
        self._check(self._lib.rmesh_backward(self._ctx, p, *ptrs))

    def forward_error(self, pixel_err, ssim_err):
        """Per-tet error statistics over the last forward_tiled's tile lists
        (lib.rs:1621-1710): (tet_err [M, 16] float32, tet_count [M, 2] int32)."""
        n = self._width * self._height
        keep = []
        ps = []
        for name, arr in (("pixel_err", pixel_err), ("ssim_err", ssim_err)):
            obj, p = _as_array(arr, np.float32, name)
            if _numel(obj) != n:
                raise ValueError(f"{name} must have {n} elements, got {_numel(obj)}")
            keep.append(obj)
            ps.append(p)
        err = np.empty((self._M, 16), np.float32)
        cnt = np.empty((self._M, 2), np.int32)
        self._check(self._lib.rmesh_forward_error(self._ctx, ps[0], ps[1], err.ctypes.data, cnt.ctypes.data))
        return err, cnt

    def train_step(self, cam_pos, vp, c2w_intrinsics, gt_image, lr_verts: float, lr_dens: float,
                   lr_grads: float, loss_type: int, lr_sh: float = 0.0) -> float:
        cam = self._cam(cam_pos, vp, c2w_intrinsics)
        self._check(self._lib.rmesh_set_lr_sh(self._ctx, float(lr_sh)))
        obj, p = _as_array(gt_image, np.float32, "gt_image")
        if _numel(obj) != 3 * self._width * self._height:
            raise ValueError("gt_image must be [H, W, 3]")
        loss = ctypes.c_float(0.0)
        self._check(self._lib.rmesh_train_step(self._ctx, ctypes.byref(cam), p, float(lr_verts), float(lr_dens),
                                               float(lr_grads), int(loss_type), ctypes.byref(loss)))
        return float(loss.value)

    def _views_args(self, cameras, gt_images, lr_verts, lr_dens, lr_grads, loss_type, lr_base, mode, lr_sh=0.0):
        n = len(cameras)
        cams = (_lib.Camera * n)()
        total = 0
        for i, c in enumerate(cameras):
            cams[i] = _camera_struct(c.cam_pos, c.vp, c.c2w_intrinsics, c.width, c.height)
            total += 3 * c.width * c.height
        if isinstance(gt_images, StagedTargets):
            if gt_images._stager._lib_stream is not self.torch_stream():
                raise ValueError("staged targets belong to another renderer or stream")
            obj, p = gt_images, None
        elif isinstance(gt_images, (list, tuple)):
            flat = np.concatenate([np.asarray(_to_numpy(g), np.float32).ravel() for g in gt_images])
            obj, p = flat, flat.ctypes.data
        else:
            obj, p = _as_array(gt_images, np.float32, "gt_images")
        if _numel(obj) != total:
            raise ValueError("gt images do not match the cameras' sizes")
        if p is None:
            p = obj._before_step()  # the renderer's stream waits for the targets' copy
        o = _lib.TrainOpts()
        o.lr_verts, o.lr_dens, o.lr_grads, o.lr_base = float(lr_verts), float(lr_dens), float(lr_grads), float(lr_base)
        o.loss_type = int(loss_type)
        o.lr_sh = float(lr_sh)
        o.mode = {"plain": _lib.MODE_PLAIN, "batched": _lib.MODE_BATCHED, "graph": _lib.MODE_GRAPH}[mode]
        return n, cams, obj, p, o

    def forward_views(self, cameras: Sequence, render_aux: bool = False, out=None):
        """Renders several cameras (``rmesh_b200.camera.Camera`` objects, any
        sizes) in one batched launch.  Returns a list of [H, W, 4] images (and
        a list of [H, W, 8 + aux_dim] aux images when ``render_aux``), each
        equal to ``forward_tiled``'s for that camera.  With ``out`` (a float32
        CUDA tensor of 4 x the cameras' total pixels) the images are written
        there back to back, without a host copy, and ``out`` is returned."""
        n = len(cameras)
        cams = (_lib.Camera * n)()
        sizes = []
        for i, c in enumerate(cameras):
            cams[i] = _camera_struct(c.cam_pos, c.vp, c.c2w_intrinsics, c.width, c.height)
            sizes.append((int(c.height), int(c.width)))
        total = sum(h * w for h, w in sizes)
        if out is not None:
            if render_aux:
                raise ValueError("out= writes the RGBA images only")
            if not (_is_torch(out) and out.is_cuda and out.dtype.is_floating_point and out.element_size() == 4
                    and out.is_contiguous() and out.numel() == 4 * total):
                raise ValueError(f"out must be a contiguous float32 CUDA tensor of {4 * total} values")
            self._check(self._lib.rmesh_forward_views(self._ctx, cams, n, out.data_ptr(), None))
            return out
        na = 8 + self._aux_dim
        rgba = np.empty(total * 4, np.float32)
        aux = np.empty(total * na, np.float32) if render_aux else None
        self._check(self._lib.rmesh_forward_views(self._ctx, cams, n, rgba.ctypes.data,
                                                  aux.ctypes.data if render_aux else None))
        imgs, auxs, o = [], [], 0
        for h, w in sizes:
            imgs.append(rgba[4 * o:4 * (o + h * w)].reshape(h, w, 4))
            if render_aux:
                auxs.append(aux[na * o:na * (o + h * w)].reshape(h, w, na))
            o += h * w
        return (imgs, auxs) if render_aux else imgs

    def train_step_views(self, cameras: Sequence, gt_images, lr_verts: float, lr_dens: float, lr_grads: float,
                         loss_type: int = 1, lr_base: float = 0.0, mode: str = "graph",
                         lr_sh: float = 0.0) -> np.ndarray:
        """One step over several cameras (``rmesh_b200.camera.Camera`` objects) with
        one Adam update.  ``gt_images``: list of [H,W,3] arrays or one flat
        array/tensor holding them back to back.  ``mode``: plain | batched | graph.
        Returns the per-view losses."""
        n, cams, keep, p, o = self._views_args(cameras, gt_images, lr_verts, lr_dens, lr_grads, loss_type,
                                               lr_base, mode, lr_sh)
        losses = np.zeros(n, np.float32)
        self._check(self._lib.rmesh_train_step_views(self._ctx, cams, n, p, ctypes.byref(o), losses.ctypes.data))
        return losses

    def accumulate_views(self, cameras: Sequence, gt_images, loss_type: int = 1, mode: str = "graph") -> np.ndarray:
        """Forward + loss + adjoint over ``cameras``; gradients land in the
        per-tet slots (see ``grad_slots``), no parameter update."""
        n, cams, keep, p, o = self._views_args(cameras, gt_images, 0.0, 0.0, 0.0, loss_type, 0.0, mode)
        losses = np.zeros(n, np.float32)
        self._check(self._lib.rmesh_accumulate_views(self._ctx, cams, n, p, ctypes.byref(o), losses.ctypes.data))
        return losses

    def autotune_tile_size(self, cameras: Sequence, gt_images, loss_type: int = 1) -> dict:
        """Times the batched forward + loss + adjoint of ``cameras`` at tile
        sizes 8, 12 and 16 with one thread per pixel (parameters unchanged),
        keeps the fastest and returns {tile_size: ms per run}."""
        n, cams, keep, p, o = self._views_args(cameras, gt_images, 0.0, 0.0, 0.0, loss_type, 0.0, "batched")
        best = ctypes.c_int32(0)
        ms = np.zeros(3, np.float32)
        self._check(self._lib.rmesh_autotune_tile_size(self._ctx, cams, n, p, ctypes.byref(o), ctypes.byref(best),
                                                       ms.ctypes.data))
        self._tile_size = int(best.value)
        return {8: float(ms[0]), 12: float(ms[1]), 16: float(ms[2])}

    def autotune(self, cameras: Sequence, gt_images, loss_type: int = 1, per_resolution: bool = True) -> dict:
        """Searches tile size x threads per tile (parameters unchanged): every
        configuration on all views, then (``per_resolution``) on the views of
        each resolution, keeping per-resolution configurations only if the mixed
        step is faster.  Returns {"grid": [{"views", "tile_size", "threads",
        "ms"}, ...], "chosen": {"default": (tile_size, threads),
        "per_resolution": {"WxH": (tile_size, threads)}}}."""
        n, cams, keep, p, o = self._views_args(cameras, gt_images, 0.0, 0.0, 0.0, loss_type, 0.0, "batched")
        cap = 6 + 6 * 16 + 1
        entries = (_lib.TuneEntry * cap)()
        got = ctypes.c_int32(0)
        self._check(self._lib.rmesh_autotune(self._ctx, cams, n, p, ctypes.byref(o), 1 if per_resolution else 0,
                                             entries, cap, ctypes.byref(got)))
        grid = []
        for e in entries[:min(int(got.value), cap)]:
            views = "all" if e.width == 0 else ("all, per-resolution configurations" if e.width < 0
                                                else f"{e.width}x{e.height}")
            grid.append({"views": views, "tile_size": int(e.tile_size), "threads": int(e.threads),
                         "ms": round(float(e.ms), 3)})
        self._tile_size, threads = self.tile_config()
        per = {}
        for c in cameras:
            key = f"{int(c.width)}x{int(c.height)}"
            cfg = self.tile_config(int(c.width), int(c.height))
            if cfg != (self._tile_size, threads):
                per[key] = cfg
        return {"grid": grid, "chosen": {"default": (self._tile_size, threads), "per_resolution": per}}

    def grad_slots(self):
        """The device gradient buffer as a flat torch CUDA tensor view: [M, 20]
        slots (density, base rgb, colour-gradient xyz, 4 x vertex xyz, pad), then,
        with SH colours, the [M, 3, nc] coefficient gradients."""
        import torch

        ptr = ctypes.c_void_p()
        n = ctypes.c_uint64()
        self._check(self._lib.rmesh_grad_slots(self._ctx, ctypes.byref(ptr), ctypes.byref(n)))

        class _View:
            __cuda_array_interface__ = {"shape": (int(n.value),), "typestr": "<f4", "data": (ptr.value, False),
                                        "version": 3, "strides": None}

        return torch.as_tensor(_View(), device="cuda")

    def apply_adam(self, lr_verts: float, lr_dens: float, lr_grads: float, lr_base: float = 0.0,
                   loss_type: int = 1, lr_sh: float = 0.0):
        o = _lib.TrainOpts()
        o.lr_verts, o.lr_dens, o.lr_grads, o.lr_base = float(lr_verts), float(lr_dens), float(lr_grads), float(lr_base)
        o.loss_type = int(loss_type)
        o.lr_sh = float(lr_sh)
        self._check(self._lib.rmesh_apply_adam(self._ctx, ctypes.byref(o)))

    # ---------------------------------------------------------- inspection
    def debug_tiles_touched(self) -> np.ndarray:
        out = np.empty(self._M, np.uint32)
        self._check(self._lib.rmesh_debug_tiles_touched(self._ctx, out.ctypes.data))
        return out

    def debug_pairs(self):
        n = ctypes.c_uint64(0)
        self._check(self._lib.rmesh_debug_pairs(self._ctx, None, None, 0, ctypes.byref(n)))
        tiles = np.empty(max(n.value, 1), np.uint32)
        tets = np.empty(max(n.value, 1), np.uint32)
        self._check(self._lib.rmesh_debug_pairs(self._ctx, tiles.ctypes.data, tets.ctypes.data, n.value,
                                                ctypes.byref(n)))
        return tiles[:n.value], tets[:n.value]

    def debug_ranges(self) -> np.ndarray:
        ts = self._tile_size
        nt = ((self._width + ts - 1) // ts) * ((self._height + ts - 1) // ts)
        out = np.empty(2 * nt, np.uint32)
        self._check(self._lib.rmesh_debug_ranges(self._ctx, out.ctypes.data, nt))
        return out

    # ----------------------------------------------------------- profiling
    def set_profiling(self, on: bool = True):
        self._check(self._lib.rmesh_set_profiling(self._ctx, 1 if on else 0))

    def stage_times(self):
        ms = np.zeros(_lib.N_STAGES, np.float32)
        launches = np.zeros(_lib.N_STAGES + 1, np.int32)
        self._check(self._lib.rmesh_stage_times(self._ctx, ms.ctypes.data, launches.ctypes.data))
        return ({k: float(v) for k, v in zip(_lib.STAGE_NAMES, ms)},
                {k: int(v) for k, v in zip(_lib.STAGE_NAMES, launches[:-1])}, int(launches[-1]))


def _numel(x) -> int:
    if _is_torch(x) or isinstance(x, StagedTargets):
        return int(x.numel())
    return int(np.asarray(x).size)
