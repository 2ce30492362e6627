"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/lib/librmesh_oracle_{f32,f64}.so`` (built by ``oracle/Makefile``)
and sequences the restated kernels the way the reference binding does:

* ``forward_tiled``  crates/rmesh-python/src/lib.rs:1041-1204
  project -> emit (sentinel-filled slots) -> stable sort -> tile ranges -> rasterize
* ``backward``       crates/rmesh-python/src/lib.rs:1894-2031
* ``train_step``     crates/rmesh-python/src/lib.rs:2405-2636
  (step += 1; Adam on vertices, densities, color_grads; base colors untouched)

Only the test tree, the smoke check and the benchmark's CPU baseline use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build() -> None:
    """Compile the oracle libraries (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(dtype: str):
    if dtype not in _LIBS:
        path = os.path.join(_HERE, "lib", f"librmesh_oracle_{dtype}.so")
        if not os.path.exists(path):
            build()
        _LIBS[dtype] = ctypes.CDLL(path)
    return _LIBS[dtype]


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctype)


class Oracle:
    """CPU restatement of the tiled path in float32 (``dtype='f32'``) or float64."""

    def __init__(self, dtype: str = "f32", threads: int = 0):
        self.dtype = dtype
        self.np = np.float32 if dtype == "f32" else np.float64
        self.rp = _f32p if dtype == "f32" else _f64p
        self.lib = _lib(dtype)
        s = "_" + dtype
        L = self.lib
        self._project = getattr(L, "orc_project" + s)
        self._emit = getattr(L, "orc_emit" + s)
        self._emit.restype = ctypes.c_int64
        self._sort = getattr(L, "orc_sort_pairs" + s)
        self._bits = getattr(L, "orc_sorting_bits" + s)
        self._ranges = getattr(L, "orc_tile_ranges" + s)
        self._raster = getattr(L, "orc_rasterize" + s)
        self._loss = getattr(L, "orc_loss" + s)
        self._loss.restype = ctypes.c_double
        self._backward = getattr(L, "orc_backward" + s)
        self._backward_aux = getattr(L, "orc_backward_aux" + s)
        self._adam = getattr(L, "orc_adam" + s)
        self._sh_backward = getattr(L, "orc_sh_backward" + s)
        rt = ctypes.c_float if dtype == "f32" else ctypes.c_double
        self._rt = rt
        self._raster.argtypes = [self.rp, _u32p, self.rp, self.rp, self.rp, _u32p, _u32p, self.rp, self.rp,
                                 self.rp, self.rp, ctypes.c_int, ctypes.c_int, ctypes.c_int, rt,
                                 self.rp, self.rp, _u32p, self.rp, ctypes.c_int]
        self._adam.argtypes = [ctypes.c_int64, self.rp, self.rp, self.rp, self.rp, ctypes.c_uint32, rt, rt, rt, rt]
        if threads > 0:
            getattr(L, "orc_set_threads" + s)(int(threads))
        self.max_threads = getattr(L, "orc_max_threads" + s)()

    # ---- helpers ----------------------------------------------------------
    def _r(self, a):
        return np.ascontiguousarray(np.asarray(a, dtype=self.np))

    @staticmethod
    def _u(a):
        return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))

    def _cam(self, cam):
        ci = np.asarray(cam.c2w_intrinsics, dtype=np.float64)
        c2w = np.concatenate([ci[0:3], ci[4:7], ci[8:11]])
        return (self._r(cam.vp), self._r(c2w), self._r(ci[12:16]), self._r(cam.cam_pos),
                int(cam.width), int(cam.height))

    @staticmethod
    def sorting_bits(num_tiles: int) -> int:
        tile_bits = 1 if num_tiles <= 1 else int(num_tiles - 1).bit_length()
        return (32 + tile_bits + 7) & ~7

    def sh_values(self, sh, f16=True):
        """Coefficient values the SH colour reads: the reference stores them as
        f16 with round-to-nearest-even (crates/rmesh-viewer/src/gpu_state.rs:60-88);
        f16=False keeps them unrounded (finite-difference checks in float64)."""
        if sh is None:
            return None
        a = np.asarray(sh, dtype=np.float32)
        if f16:
            a = a.astype(np.float16).astype(np.float32)
        return self._r(a)

    # ---- stages -----------------------------------------------------------
    def project(self, scene, cam, tile_size=12, sh=None, sh_degree=0):
        """sh: coefficient values [M*3*nc] as read by the shader (see sh_values)."""
        v, idx = self._r(scene["vertices"]), self._u(scene["indices"])
        m = idx.size // 4
        vp, c2w, intr, cp, W, H = self._cam(cam)
        visible = np.zeros(m, dtype=np.uint8)
        tt = np.zeros(m, dtype=np.uint32)
        colors = np.zeros(3 * m, dtype=self.np)
        shp = None if sh is None else self._r(sh)
        self._project(ctypes.c_int64(m), _ptr(v, self.rp), _ptr(idx, _u32p), _ptr(self._r(scene["densities"]), self.rp),
                      _ptr(self._r(scene["color_grads"]), self.rp), _ptr(self._r(scene["circumdata"]), self.rp),
                      _ptr(self._r(scene["base_colors"]), self.rp), _ptr(shp, self.rp), ctypes.c_int(sh_degree),
                      _ptr(vp, self.rp), _ptr(cp, self.rp), ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(tile_size),
                      _ptr(visible, _u8p), _ptr(tt, _u32p), _ptr(colors, self.rp))
        return visible, tt, colors

    def emit(self, scene, cam, visible, tiles_touched, tile_size=12):
        v, idx = self._r(scene["vertices"]), self._u(scene["indices"])
        m = idx.size // 4
        vp, c2w, intr, cp, W, H = self._cam(cam)
        cap = int(tiles_touched[visible.astype(bool)].astype(np.int64).sum())
        lo = np.zeros(max(cap, 1), dtype=np.uint32)
        hi = np.zeros(max(cap, 1), dtype=np.uint32)
        vals = np.zeros(max(cap, 1), dtype=np.uint32)
        emitted = ctypes.c_int64(0)
        P = self._emit(ctypes.c_int64(m), _ptr(v, self.rp), _ptr(idx, _u32p), _ptr(self._r(scene["circumdata"]), self.rp),
                       _ptr(vp, self.rp), _ptr(cp, self.rp), ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(tile_size),
                       _ptr(np.ascontiguousarray(visible), _u8p), _ptr(self._u(tiles_touched), _u32p),
                       _ptr(lo, _u32p), _ptr(hi, _u32p), _ptr(vals, _u32p), ctypes.c_int64(cap),
                       ctypes.byref(emitted))
        assert P == cap
        return lo[:P], hi[:P], vals[:P], int(emitted.value)

    def sort_pairs(self, lo, hi, vals, num_tiles):
        lo, hi, vals = lo.copy(), hi.copy(), vals.copy()
        self._sort(ctypes.c_int64(lo.size), ctypes.c_int(self.sorting_bits(num_tiles)), _ptr(lo, _u32p),
                   _ptr(hi, _u32p), _ptr(vals, _u32p))
        return lo, hi, vals

    def tile_ranges(self, hi_sorted, num_tiles):
        ranges = np.zeros(2 * num_tiles, dtype=np.uint32)
        self._ranges(ctypes.c_int64(hi_sorted.size), _ptr(self._u(hi_sorted), _u32p), _ptr(ranges, _u32p))
        return ranges

    def rasterize(self, scene, cam, colors, vals, ranges, tile_size=12, min_t=0.0, aux=False, stats=False,
                  aux_data=None):
        """aux_data: optional [M * aux_dim] custom channels composited after the 8 fixed aux ones."""
        vp, c2w, intr, cp, W, H = self._cam(cam)
        m = scene["indices"].size // 4
        aux_dim = 0 if aux_data is None else int(np.asarray(aux_data).size // m)
        rgba = np.zeros(H * W * 4, dtype=self.np)
        auxb = np.zeros(H * W * (8 + aux_dim), dtype=self.np) if aux else None
        st = np.zeros(H * W * 4, dtype=np.uint32) if stats else None
        self._raster(_ptr(self._r(scene["vertices"]), self.rp), _ptr(self._u(scene["indices"]), _u32p),
                     _ptr(self._r(colors), self.rp), _ptr(self._r(scene["densities"]), self.rp),
                     _ptr(self._r(scene["color_grads"]), self.rp), _ptr(self._u(vals), _u32p),
                     _ptr(self._u(ranges), _u32p), _ptr(vp, self.rp), _ptr(c2w, self.rp), _ptr(intr, self.rp),
                     _ptr(cp, self.rp), W, H, tile_size, self._rt(min_t), _ptr(rgba, self.rp), _ptr(auxb, self.rp),
                     _ptr(st, _u32p), _ptr(None if aux_data is None else self._r(aux_data), self.rp), aux_dim)
        out = {"image": rgba.reshape(H, W, 4)}
        if aux:
            out["aux"] = auxb.reshape(H, W, 8 + aux_dim)
        if stats:
            out["stats"] = st.reshape(H, W, 4)
        return out

    def loss(self, rendered, gt, loss_type=1):
        rendered = self._r(rendered)
        H, W = rendered.shape[0], rendered.shape[1]
        dl = np.zeros(H * W * 4, dtype=self.np)
        val = self._loss(ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(loss_type), _ptr(rendered, self.rp),
                         _ptr(self._r(gt), self.rp), _ptr(dl, self.rp))
        return float(val), dl.reshape(H, W, 4)

    def backward_raw(self, scene, cam, colors, vals, ranges, dl, rendered, tile_size=12, threads=1,
                     aux_data=None, dl_aux=None):
        """With aux_data [M*aux_dim] and dl_aux [H*W*aux_dim] also returns
        d_aux_data (the custom aux channels' adjoint, see orc_backward_aux)."""
        vp, c2w, intr, cp, W, H = self._cam(cam)
        n = scene["vertices"].size
        m = scene["indices"].size // 4
        dv = np.zeros(n, dtype=self.np)
        dd = np.zeros(m, dtype=self.np)
        dg = np.zeros(3 * m, dtype=self.np)
        db = np.zeros(3 * m, dtype=self.np)
        aux_dim = 0 if aux_data is None or dl_aux is None else int(np.asarray(aux_data).size // m)
        da = np.zeros(max(aux_dim, 1) * m, dtype=self.np)
        self._backward_aux(_ptr(self._r(scene["vertices"]), self.rp), _ptr(self._u(scene["indices"]), _u32p),
                           _ptr(self._r(colors), self.rp), _ptr(self._r(scene["densities"]), self.rp),
                           _ptr(self._r(scene["color_grads"]), self.rp), _ptr(self._u(vals), _u32p),
                           _ptr(self._u(ranges), _u32p), _ptr(vp, self.rp), _ptr(c2w, self.rp), _ptr(intr, self.rp),
                           _ptr(cp, self.rp), ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(tile_size),
                           _ptr(self._r(dl), self.rp), _ptr(self._r(rendered), self.rp), _ptr(dv, self.rp),
                           _ptr(dd, self.rp), _ptr(dg, self.rp), _ptr(db, self.rp), ctypes.c_int(threads),
                           _ptr(self._r(aux_data) if aux_dim else None, self.rp), ctypes.c_int(aux_dim),
                           _ptr(self._r(dl_aux) if aux_dim else None, self.rp), _ptr(da, self.rp))
        out = {"d_vertices": dv, "d_densities": dd, "d_color_grads": dg, "d_base_colors": db}
        if aux_dim:
            out["d_aux_data"] = da
        return out

    def error_stats(self, scene, cam, fwd, pixel_err, ssim_err, tile_size=12, min_t=0.0):
        """Per-tet error statistics (error_tiled_compute.wgsl:90-373) over the
        tile lists of the forward ``fwd``: (tet_err [M, 16] f64, tet_count [M, 2] i32)."""
        vp, c2w, intr, cp, W, H = self._cam(cam)
        m = scene["indices"].size // 4
        err = np.zeros(16 * m, np.float64)
        cnt = np.zeros(2 * m, np.int32)
        fn = getattr(self.lib, "orc_error_stats_" + self.dtype)
        fn(_ptr(self._r(scene["vertices"]), self.rp), _ptr(self._u(scene["indices"]), _u32p),
           _ptr(self._r(scene["densities"]), self.rp), _ptr(self._u(fwd["vals"]), _u32p),
           _ptr(self._u(fwd["ranges"]), _u32p), _ptr(vp, self.rp), _ptr(c2w, self.rp), _ptr(intr, self.rp),
           _ptr(cp, self.rp), ctypes.c_int(W), ctypes.c_int(H), ctypes.c_int(tile_size), self._rt(min_t),
           _ptr(self._r(pixel_err), self.rp), _ptr(self._r(ssim_err), self.rp), _ptr(err, _f64p),
           _ptr(cnt, ctypes.POINTER(ctypes.c_int32)))
        return err.reshape(m, 16), cnt.reshape(m, 2)

    def rmesh_decode(self, raw: bytes) -> dict:
        """crates/rmesh-data/src/lib.rs:247-393 on decompressed .rmesh bytes."""
        buf = np.frombuffer(raw, dtype=np.uint8)
        hdr = np.zeros(4, np.uint32)
        if getattr(self.lib, "orc_rmesh_header_" + self.dtype)(_ptr(buf, _u8p), ctypes.c_int64(buf.size),
                                                                _ptr(hdr, _u32p)) != 0:
            raise ValueError("truncated .rmesh header")
        n, m, deg, _ = (int(x) for x in hdr)
        nc = (deg + 1) ** 2
        out = {"start_pose": np.zeros(7, np.float32), "vertices": np.zeros(3 * n, np.float32),
               "indices": np.zeros(4 * m, np.uint32), "densities": np.zeros(m, np.float32),
               "sh_coeffs": np.zeros(3 * nc * m, np.float32), "color_grads": np.zeros(3 * m, np.float32),
               "circumdata": np.zeros(4 * m, np.float32)}
        fn = getattr(self.lib, "orc_rmesh_decode_" + self.dtype)
        fn.restype = ctypes.c_int64
        fp = lambda k: _ptr(out[k], _f32p)
        end = fn(_ptr(buf, _u8p), ctypes.c_int64(buf.size), fp("start_pose"), fp("vertices"),
                 _ptr(out["indices"], _u32p), fp("densities"), fp("sh_coeffs"), fp("color_grads"), fp("circumdata"))
        if end < 0:
            raise ValueError("truncated .rmesh file")
        out["sh_degree"] = deg
        return out

    def adam(self, params, grads, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        """In place on float arrays of this oracle's dtype."""
        self._adam(ctypes.c_int64(params.size), _ptr(params, self.rp), _ptr(self._r(grads), self.rp),
                   _ptr(m, self.rp), _ptr(v, self.rp), ctypes.c_uint32(step), self._rt(lr), self._rt(beta1),
                   self._rt(beta2), self._rt(eps))

    # ---- host sequencing --------------------------------------------------
    def forward_tiled(self, scene, cam, tile_size=12, min_t=0.0, aux=False, stats=False,
                      sh=None, sh_degree=0, aux_data=None):
        """lib.rs:1041-1204.  Returns the image plus every intermediate buffer.
        sh: coefficient values (see sh_values) selecting the SH colour branch."""
        W, H = int(cam.width), int(cam.height)
        tiles_x = (W + tile_size - 1) // tile_size
        tiles_y = (H + tile_size - 1) // tile_size
        num_tiles = tiles_x * tiles_y
        visible, tt, colors = self.project(scene, cam, tile_size, sh, sh_degree)
        lo, hi, vals, emitted = self.emit(scene, cam, visible, tt, tile_size)
        slo, shi, svals = self.sort_pairs(lo, hi, vals, num_tiles)
        ranges = self.tile_ranges(shi, num_tiles)
        out = self.rasterize(scene, cam, colors, svals, ranges, tile_size, min_t, aux, stats, aux_data)
        out.update(visible=visible, tiles_touched=tt, colors=colors, key_lo=slo, key_hi=shi, vals=svals,
                   ranges=ranges, P=int(lo.size), emitted=emitted, num_tiles=num_tiles,
                   unsorted=(lo, hi, vals))
        return out

    def backward(self, scene, cam, dl_d_image, fwd, tile_size=12, threads=1, sh=None, sh_degree=0,
                 aux_data=None, dl_aux=None):
        """lib.rs:1894-2031 (the sort it redoes equals the forward's).  With sh
        (the coefficient values of the forward), the colour gradient continues
        through the SH colour: d_sh is added, d_vertices and d_color_grads gain
        the colour's dependence on them, and d_base_colors is zero."""
        g = self.backward_raw(scene, cam, fwd["colors"], fwd["vals"], fwd["ranges"],
                              np.asarray(dl_d_image).reshape(-1), fwd["image"].reshape(-1), tile_size, threads,
                              aux_data=aux_data, dl_aux=None if dl_aux is None else np.asarray(dl_aux).reshape(-1))
        if sh is not None:
            g["d_sh"] = self.sh_backward(scene, cam, sh, sh_degree, fwd["visible"], g["d_base_colors"],
                                         g["d_vertices"], g["d_color_grads"])
            g["d_base_colors"] = np.zeros_like(g["d_base_colors"])
        return g

    def sh_backward(self, scene, cam, sh, sh_degree, visible, d_colors, d_vertices, d_color_grads):
        """Adjoint of the SH colour; adds into d_vertices / d_color_grads in place."""
        m = scene["indices"].size // 4
        nc = (sh_degree + 1) ** 2
        d_sh = np.zeros(3 * nc * m, dtype=self.np)
        cp = self._r(cam.cam_pos)
        self._sh_backward(ctypes.c_int64(m), _ptr(self._r(scene["vertices"]), self.rp),
                          _ptr(self._u(scene["indices"]), _u32p), _ptr(self._r(scene["color_grads"]), self.rp),
                          _ptr(self._r(sh), self.rp), ctypes.c_int(sh_degree), _ptr(cp, self.rp),
                          _ptr(np.ascontiguousarray(visible, dtype=np.uint8), _u8p), _ptr(self._r(d_colors), self.rp),
                          _ptr(d_sh, self.rp), _ptr(d_vertices, self.rp), _ptr(d_color_grads, self.rp))
        return d_sh

    def loss_value(self, scene, cam, gt, loss_type=1, tile_size=12):
        fwd = self.forward_tiled(scene, cam, tile_size)
        val, _ = self.loss(fwd["image"], gt, loss_type)
        return val


class OracleTrainer:
    """lib.rs:2405-2636 on the CPU: one view per step, Adam on three groups
    (four with SH colours: use_sh adds the coefficients, learning rate lr_sh)."""

    def __init__(self, scene, dtype="f32", tile_size=12, use_sh=False):
        self.o = Oracle(dtype)
        self.scene = {k: (np.array(v, dtype=self.o.np) if k in ("vertices", "densities", "color_grads",
                                                                "base_colors", "circumdata") else v)
                      for k, v in scene.items()}
        self.use_sh = use_sh
        groups = ["vertices", "densities", "color_grads"]
        if use_sh:
            self.sh = np.array(scene["sh_coeffs"], dtype=np.float32)  # fp32 master values
            self.sh_degree = int(scene["sh_degree"])
            self.m_sh = np.zeros_like(self.sh, dtype=self.o.np)
            self.v_sh = np.zeros_like(self.sh, dtype=self.o.np)
        self.tile_size = tile_size
        self.step = 0
        z = lambda k: np.zeros_like(self.scene[k])
        self.m = {k: z(k) for k in groups}
        self.v = {k: z(k) for k in groups}

    def train_step(self, cam, gt, lr_verts, lr_dens, lr_grads, loss_type=1, lr_sh=0.0):
        loss, fwd, g = self._view_grads(cam, gt, loss_type, threads=1)
        self._adam_all(g, lr_verts, lr_dens, lr_grads, lr_sh)
        return loss, fwd, g

    def train_step_views(self, cams, gts, lr_verts, lr_dens, lr_grads, loss_type=1, lr_sh=0.0, threads=1):
        """The multi-view step of the B200 library (no reference counterpart): the
        gradient of the sum of the per-view losses (each the single-view loss of
        lib.rs:2405-2636 over its own pixels), then one Adam update.  Returns the
        per-view losses."""
        losses, total = [], None
        for cam, gt in zip(cams, gts):
            loss, _, g = self._view_grads(cam, gt, loss_type, threads)
            losses.append(loss)
            total = g if total is None else {k: total[k] + g[k] for k in total}
        self._adam_all(total, lr_verts, lr_dens, lr_grads, lr_sh)
        return np.array(losses)

    def _view_grads(self, cam, gt, loss_type, threads):
        shv = self.o.sh_values(self.sh) if self.use_sh else None
        deg = self.sh_degree if self.use_sh else 0
        fwd = self.o.forward_tiled(self.scene, cam, self.tile_size, sh=shv, sh_degree=deg)
        loss, dl = self.o.loss(fwd["image"], gt, loss_type)
        g = self.o.backward(self.scene, cam, dl, fwd, self.tile_size, threads=threads, sh=shv, sh_degree=deg)
        return loss, fwd, g

    def _adam_all(self, g, lr_verts, lr_dens, lr_grads, lr_sh):
        self.step += 1
        for key, gk, lr in (("vertices", "d_vertices", lr_verts), ("densities", "d_densities", lr_dens),
                            ("color_grads", "d_color_grads", lr_grads)):
            self.o.adam(self.scene[key], g[gk], self.m[key], self.v[key], self.step, lr)
        if self.use_sh:
            p = self.sh.astype(self.o.np)
            self.o.adam(p, g["d_sh"], self.m_sh, self.v_sh, self.step, lr_sh)
            self.sh = p.astype(np.float32)
