""".rmesh scene files (crates/rmesh-data/src/lib.rs:142-393) -> device buffers.

A .rmesh file is gzip-compressed (or raw) little-endian binary:

    u32 N, M, sh_degree, k            header
    f32 pose[8]                       x, y, z, qx, qy, qz, qw, pad
    f32 vertices[3N]; u32 indices[4M]
    u8  log-densities[M]              density = exp((u8 - 100) / 20)
    (align 4)
    f16 SH mean[D], basis[k'][D], weights[M][k']   D = 3 (deg+1)^2, k' = min(k, D)
    (align 4)
    f16 colour gradients[3M]          zeros if a tagged "RMTX" section starts here
                                      instead; zero-padded if the file is short

The host (this module) decompresses, reads the header and slices the
sections without copying; the sections are uploaded as they are and decoded on
the device by ``rmesh_decode_scene`` (densities, f16 conversion, PCA
decompression of the SH coefficients, double-precision circumspheres).
Tagged PBR extension sections after the gradients are not read.
"""
from __future__ import annotations

import ctypes
import gzip
import os

import numpy as np

from . import _lib

__all__ = ["read_rmesh_bytes", "parse_rmesh_sections", "load_rmesh"]

_TAGGED_MAGIC = 0x524D5458  # "RMTX"
_HEADER_BYTES = 48


def read_rmesh_bytes(source) -> bytes:
    """File path, bytes or file object -> decompressed bytes (gzip is detected
    by its magic, as the reference's decompress_gzip does, lib.rs:152-171)."""
    if isinstance(source, (str, os.PathLike)):
        with open(source, "rb") as f:
            data = f.read()
    elif hasattr(source, "read"):
        data = source.read()
    else:
        data = bytes(source)
    if len(data) >= 2 and data[0] == 0x1F and data[1] == 0x8B:
        data = gzip.decompress(data)
    return data


def _align4(x: int) -> int:
    return (x + 3) & ~3


def parse_rmesh_sections(raw: bytes) -> dict:
    """Header fields and zero-copy numpy views of every section of the
    decompressed file (lib.rs:247-330).  Raises ValueError on a short file."""
    buf = np.frombuffer(raw, dtype=np.uint8)
    if buf.size < _HEADER_BYTES:
        raise ValueError(".rmesh file shorter than its header")
    n, m, deg, k = (int(x) for x in buf[:16].view(np.uint32))
    if deg > 3:
        raise ValueError(f".rmesh SH degree {deg} is not 0..3")
    pose = buf[16:44].view(np.float32).copy()
    nc = (deg + 1) ** 2
    d = 3 * nc
    kk = min(k, d)
    off = _HEADER_BYTES
    need = off + 12 * n + 16 * m + m
    if buf.size < need:
        raise ValueError(".rmesh file truncated in its geometry")
    out = {"n_vertices": n, "n_tets": m, "sh_degree": deg, "k_components": k, "start_pose": pose}
    out["vertices"] = buf[off:off + 12 * n].view(np.float32)
    off += 12 * n
    out["indices"] = buf[off:off + 16 * m].view(np.uint32)
    off += 16 * m
    out["log_densities"] = buf[off:off + m]
    off = _align4(off + m)
    sh_bytes = 2 * (d + kk * d + m * kk)
    if buf.size < off + sh_bytes:
        raise ValueError(".rmesh file truncated in its SH section")
    out["sh_mean"] = buf[off:off + 2 * d].view(np.uint16)
    off += 2 * d
    out["sh_basis"] = buf[off:off + 2 * kk * d].view(np.uint16)
    off += 2 * kk * d
    out["sh_weights"] = buf[off:off + 2 * m * kk].view(np.uint16)
    off = _align4(off + 2 * m * kk)
    ng = 3 * m
    if off + 4 <= buf.size and int(buf[off:off + 4].view(np.uint32)[0]) == _TAGGED_MAGIC:
        out["color_grads_f16"] = None
    else:
        avail = min(ng, (buf.size - off) // 2)
        g = np.zeros(ng, np.uint16)
        g[:avail] = buf[off:off + 2 * avail].view(np.uint16)
        out["color_grads_f16"] = g
    return out


def load_rmesh(source, device="cuda"):
    """Loads a .rmesh scene onto a CUDA device.  Returns a dict of torch CUDA
    tensors vertices [3N], indices [4M] (int32 storage of the u32 ids),
    densities [M], color_grads [3M], circumdata [4M], sh_coeffs [M*3*nc], plus
    sh_degree and start_pose -- the arguments of RMeshRenderer (base_colors,
    which the file does not hold, are the DC term's colour 0.5 + C0 * sh0)."""
    import torch

    sec = parse_rmesh_sections(read_rmesh_bytes(source))
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError("load_rmesh decodes on a CUDA device")
    lib = _lib.load()
    n, m, deg = sec["n_vertices"], sec["n_tets"], sec["sh_degree"]
    nc = (deg + 1) ** 2

    def up(a, dtype):
        a = np.ascontiguousarray(a).view(dtype)
        if not a.flags.writeable:  # a view of the immutable file bytes
            a = a.copy()
        return torch.from_numpy(a).to(dev)

    verts = up(sec["vertices"], np.float32)
    idx = up(sec["indices"], np.int32)
    logd = up(sec["log_densities"], np.uint8)
    mean = up(sec["sh_mean"], np.int16)
    basis = up(sec["sh_basis"], np.int16) if sec["sh_basis"].size else torch.zeros(1, dtype=torch.int16, device=dev)
    weights = up(sec["sh_weights"], np.int16) if sec["sh_weights"].size else torch.zeros(1, dtype=torch.int16,
                                                                                         device=dev)
    grads16 = None if sec["color_grads_f16"] is None else up(sec["color_grads_f16"], np.int16)
    dens = torch.empty(m, dtype=torch.float32, device=dev)
    grads = torch.empty(3 * m, dtype=torch.float32, device=dev)
    sh = torch.empty(3 * nc * m, dtype=torch.float32, device=dev)
    circ = torch.empty(4 * m, dtype=torch.float32, device=dev)
    ps = _lib.PackedScene()
    ps.n_vertices, ps.n_tets, ps.sh_degree, ps.k_components = n, m, deg, sec["k_components"]
    ps.vertices, ps.indices, ps.log_densities = verts.data_ptr(), idx.data_ptr(), logd.data_ptr()
    ps.sh_mean, ps.sh_basis, ps.sh_weights = mean.data_ptr(), basis.data_ptr(), weights.data_ptr()
    ps.color_grads = None if grads16 is None else grads16.data_ptr()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream().cuda_stream
        rc = lib.rmesh_decode_scene(ctypes.byref(ps), dens.data_ptr(), grads.data_ptr(), sh.data_ptr(),
                                    circ.data_ptr(), ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"rmesh_decode_scene failed with status {rc}")
        torch.cuda.current_stream().synchronize()
    from .scenes import SH_C0

    base = (0.5 + SH_C0 * sh.view(m, 3, nc)[:, :, 0]).reshape(-1).contiguous()
    return {"vertices": verts, "indices": idx, "densities": dens, "color_grads": grads, "circumdata": circ,
            "sh_coeffs": sh, "sh_degree": deg, "base_colors": base, "start_pose": sec["start_pose"]}
