"""PyTorch autograd integration (crates/rmesh-python/python/rmesh_wgpu/autograd.py:15-151).

``RMeshForward.apply(renderer, cam_pos, vp, c2w_intrinsics, vertices,
base_colors, densities, color_grads, render_mode="tiled")`` renders a
[H, W, 4] premultiplied RGBA image; its backward returns gradients for the four
parameter tensors and ``None`` for the rest, exactly as the reference does.
An optional trailing ``sh_coeffs`` tensor (a renderer built with SH
coefficients; no counterpart in the reference's binding) is uploaded before
the render and receives its gradient.

When the parameters are CUDA tensors, parameters, image and gradients move
device-to-device through the C ABI (no numpy round trip); CPU tensors take the
host path like the reference.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn as nn

from .renderer import RMeshRenderer

__all__ = ["RMeshForward", "RMeshModule"]


class RMeshForward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer, cam_pos, vp, c2w_intrinsics, vertices, base_colors, densities, color_grads,
                render_mode="tiled", sh_coeffs=None):
        if render_mode != "tiled":
            raise ValueError("only render_mode='tiled' is provided by this renderer")
        if (sh_coeffs is not None) != (renderer.sh_degree >= 0):
            raise ValueError("pass sh_coeffs exactly when the renderer was built with SH coefficients")
        renderer.update_params(vertices.detach().reshape(-1), base_colors.detach().reshape(-1),
                               densities.detach().reshape(-1), color_grads.detach().reshape(-1),
                               None if sh_coeffs is None else sh_coeffs.detach().reshape(-1))
        ctx.renderer = renderer
        ctx.has_sh = sh_coeffs is not None
        saved = (vertices, base_colors, densities, color_grads) + ((sh_coeffs,) if ctx.has_sh else ())
        ctx.save_for_backward(*saved)
        if vertices.is_cuda:
            out = torch.empty((renderer.height, renderer.width, 4), dtype=torch.float32, device=vertices.device)
            renderer.forward_tiled_into(cam_pos, vp, c2w_intrinsics, out)
            return out
        image = renderer.forward_tiled(cam_pos, vp, c2w_intrinsics)
        return torch.from_numpy(image.copy()).to(vertices.device)

    @staticmethod
    def backward(ctx, grad_output):
        vertices, base_colors, densities, color_grads = ctx.saved_tensors[:4]
        sh = ctx.saved_tensors[4] if ctx.has_sh else None
        r = ctx.renderer
        dsh = None
        if vertices.is_cuda:
            g = grad_output.detach().to(torch.float32).contiguous()
            dv = torch.empty_like(vertices.reshape(-1))
            db = torch.empty_like(base_colors.reshape(-1))
            dd = torch.empty_like(densities.reshape(-1))
            dg = torch.empty_like(color_grads.reshape(-1))
            r.backward_into(g, dv, dd, db, dg)
            if sh is not None:
                dsh = r.sh_grad_into(torch.empty_like(sh.reshape(-1))).view_as(sh)
        else:
            grads = r.backward(grad_output.detach().cpu().numpy().astype(np.float32))
            dev = vertices.device
            dv = torch.from_numpy(grads["d_vertices"].copy()).to(dev)
            db = torch.from_numpy(grads["d_base_colors"].copy()).to(dev)
            dd = torch.from_numpy(grads["d_densities"].copy()).to(dev)
            dg = torch.from_numpy(grads["d_color_grads"].copy()).to(dev)
            if sh is not None:
                dsh = torch.from_numpy(grads["d_sh_coeffs"].copy()).to(dev).view_as(sh)
        return (None, None, None, None, dv.view_as(vertices), db.view_as(base_colors), dd.view_as(densities),
                dg.view_as(color_grads), None, dsh)


class RMeshModule(nn.Module):
    """nn.Module holding the four learnable parameter groups plus a renderer
    (autograd.py:79-151).  ``device='cuda'`` keeps the parameters on the GPU.
    ``sh_coeffs`` adds a fifth group and colours the mesh by SH."""

    def __init__(self, vertices: np.ndarray, indices: np.ndarray, base_colors: np.ndarray, densities: np.ndarray,
                 color_grads: np.ndarray, circumdata: np.ndarray, width: int, height: int, device=None,
                 tile_size: int = 12, sh_coeffs=None, sh_degree: int | None = None):
        super().__init__()
        dev = torch.device(device) if device is not None else torch.device("cpu")
        self.vertices = nn.Parameter(torch.tensor(np.asarray(vertices).ravel(), dtype=torch.float32, device=dev))
        self.base_colors = nn.Parameter(torch.tensor(np.asarray(base_colors).ravel(), dtype=torch.float32,
                                                     device=dev))
        self.densities = nn.Parameter(torch.tensor(np.asarray(densities).ravel(), dtype=torch.float32, device=dev))
        self.color_grads = nn.Parameter(torch.tensor(np.asarray(color_grads).ravel(), dtype=torch.float32,
                                                     device=dev))
        self._indices = np.asarray(indices).ravel().astype(np.uint32)
        self._circumdata = np.asarray(circumdata).ravel().astype(np.float32)
        self._width = width
        self._height = height
        self.sh_coeffs = None
        if sh_coeffs is not None:
            self.sh_coeffs = nn.Parameter(torch.tensor(np.asarray(sh_coeffs).ravel(), dtype=torch.float32,
                                                       device=dev))
        self.renderer = RMeshRenderer(np.asarray(vertices).ravel().astype(np.float32), self._indices,
                                      np.asarray(base_colors).ravel().astype(np.float32),
                                      np.asarray(densities).ravel().astype(np.float32),
                                      np.asarray(color_grads).ravel().astype(np.float32), self._circumdata,
                                      width, height, tile_size=tile_size,
                                      sh_coeffs=None if sh_coeffs is None else
                                      np.asarray(sh_coeffs).ravel().astype(np.float32), sh_degree=sh_degree)

    def forward(self, cam_pos, vp, c2w_intrinsics, render_mode="tiled"):
        return RMeshForward.apply(self.renderer, cam_pos, vp, c2w_intrinsics, self.vertices, self.base_colors,
                                  self.densities, self.color_grads, render_mode, self.sh_coeffs)
