// Per-tet stage: record packing, projection, culling, tile counting, depth keys
// and deterministic compaction of the tile-touching tets of every view.
//
// Reference: crates/rmesh-render/src/wgsl/project_compute.wgsl:88-325 (cull,
// tiles_touched, colours) and tile_gen_scan_compute.wgsl:135-143 (the
// circumsphere depth key used for the tile sort).  The reference compacts with
// atomicAdd (project_compute.wgsl:181); here every (tet, view) item keeps its
// own slot and only the sort keys are compacted, by a chained scan in item
// order, so downstream order is deterministic.
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"

namespace rm {

// Per-tet record, view independent, rebuilt whenever parameters change.
// 64 bytes: a = (v0, density), b = (v1, g.x), c = (v2, g.y), d = (v3, g.z).
struct __align__(16) TetRec {
  float4 a, b, c, d;
};

__global__ void __launch_bounds__(256) build_records_kernel(int M, const float* __restrict__ verts,
                                                            const uint4* __restrict__ idx4,
                                                            const float* __restrict__ dens,
                                                            const float* __restrict__ cgrad,
                                                            const float* __restrict__ base,
                                                            TetRec* __restrict__ rec, float4* __restrict__ color4) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  uint4 q = idx4[t];
  float g0 = cgrad[3 * t], g1 = cgrad[3 * t + 1], g2 = cgrad[3 * t + 2];
  TetRec r;
  r.a = make_float4(verts[3 * q.x], verts[3 * q.x + 1], verts[3 * q.x + 2], dens[t]);
  r.b = make_float4(verts[3 * q.y], verts[3 * q.y + 1], verts[3 * q.y + 2], g0);
  r.c = make_float4(verts[3 * q.z], verts[3 * q.z + 1], verts[3 * q.z + 2], g1);
  r.d = make_float4(verts[3 * q.w], verts[3 * q.w + 1], verts[3 * q.w + 2], g2);
  rec[t] = r;
  if (color4) color4[t] = make_float4(base[3 * t], base[3 * t + 1], base[3 * t + 2], 0.0f);
}

// Conservative scanline over tile rows (project_compute.wgsl:202-259 ==
// tile_gen_scan_compute.wgsl:119-201), exact arithmetic.  tile_range gives a
// tet's clamped pixel box in tiles (false when it is empty), tile_row_span one
// tile row's [tx0, tx1] (false when the row is empty); scanline_tiles calls
// f(ty, tx0, tx1) for every tile row with a non-empty clamped span.
struct TileBox {
  uint32_t min_x, max_x, min_y, max_y;
};
__device__ __forceinline__ bool tile_range(const float px[4], const float py[4], float W, float H, uint32_t TS,
                                           TileBox& tb) {
  const float pix_min_x = fmaxf(fminf(fminf(px[0], px[1]), fminf(px[2], px[3])), 0.0f);
  const float pix_max_x = fminf(fmaxf(fmaxf(px[0], px[1]), fmaxf(px[2], px[3])), fs(W, 1.0f));
  const float pix_min_y = fmaxf(fminf(fminf(py[0], py[1]), fminf(py[2], py[3])), 0.0f);
  const float pix_max_y = fminf(fmaxf(fmaxf(py[0], py[1]), fmaxf(py[2], py[3])), fs(H, 1.0f));
  if (pix_min_x > pix_max_x || pix_min_y > pix_max_y) return false;
  const float T = (float)TS;
  const uint32_t tiles_x_total = __float2uint_rz(ceilf(fdv(W, T)));
  tb.min_x = __float2uint_rz(fdv(pix_min_x, T));
  tb.max_x = min(__float2uint_rz(fdv(pix_max_x, T)), tiles_x_total - 1u);
  tb.min_y = __float2uint_rz(fdv(pix_min_y, T));
  tb.max_y = min(__float2uint_rz(fdv(pix_max_y, T)), __float2uint_rz(ceilf(fdv(H, T))) - 1u);
  return true;
}
__device__ __forceinline__ bool tile_row_span(const float px[4], const float py[4], uint32_t TS, const TileBox& tb,
                                              uint32_t ty, uint32_t& tx0, uint32_t& tx1) {
  const float T = (float)TS;
  const int ei[6] = {0, 0, 0, 1, 1, 2};
  const int ej[6] = {1, 2, 3, 2, 3, 3};
  float xl = 1e10f, xr = -1e10f;
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const float yi = py[ei[e]], yj = py[ej[e]], xi = px[ei[e]], xj = px[ej[e]];
#pragma unroll
    for (uint32_t b = 0; b < 2; ++b) {
      const float ytest = fm((float)(ty + b), T);
      if ((yi <= ytest && yj > ytest) || (yj <= ytest && yi > ytest)) {
        const float t = fdv(fs(ytest, yi), fs(yj, yi));
        const float x = fa(xi, fm(t, fs(xj, xi)));
        xl = fminf(xl, x);
        xr = fmaxf(xr, x);
      }
    }
  }
  const float band_lo = fm((float)ty, T), band_hi = fm((float)(ty + 1u), T);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    if (py[v] >= band_lo && py[v] <= band_hi) {
      xl = fminf(xl, px[v]);
      xr = fmaxf(xr, px[v]);
    }
  }
  if (!(xl <= xr)) return false;
  tx0 = __float2uint_rz(fmaxf(floorf(fdv(xl, T)), 0.0f));
  tx1 = __float2uint_rz(fmaxf(floorf(fdv(xr, T)), 0.0f));
  tx0 = min(max(tx0, tb.min_x), tb.max_x);
  tx1 = min(max(tx1, tb.min_x), tb.max_x);
  return true;
}
template <class F>
__device__ __forceinline__ void scanline_tiles(const float px[4], const float py[4], float W, float H, uint32_t TS,
                                               F&& f) {
  TileBox tb;
  if (!tile_range(px, py, W, H, TS, tb)) return;
  for (uint32_t ty = tb.min_y; ty <= tb.max_y; ++ty) {
    uint32_t tx0, tx1;
    if (tile_row_span(px, py, TS, tb, ty, tx0, tx1)) f(ty, tx0, tx1);
  }
}

// Per-(view, visible tet) record consumed by the tile kernel: everything a
// tile needs about a tet that depends only on the tet and the view, computed
// once per view instead of once per (tile, tet) pair.  144 bytes (TMA-sized).
//   nrm[f]  inward normal of face f, n = cross(vc - va, vb - va) flipped toward
//           the opposite vertex, and num = dot(n, va - cam), explicitly rounded
//           (rasterize_compute.wgsl:301-314, 360-372)
//   cb      colour + dot(g, cam - v0) (the base colour at the camera, :395-396), density
//   gm      colour gradient g; w = face flip bits (bit f) | behind (bit 4)
//   px, py  pixel-space vertex projections (c.x/c.w+1)*W/2, (1-c.y/c.w)*H/2 (:163-166)
//   meta    tet id, the entry's own index (its per-view colour-gradient slot)
struct __align__(16) TetView {
  float4 nrm[4];
  float4 cb;
  float4 gm;
  float4 px;
  float4 py;
  uint4 meta;
};

__device__ __forceinline__ void write_tet_view(TetView* dst, const TetRec& r, const float4 col, const ViewParams& V,
                                               uint32_t tet, uint32_t j) {
  const float4 vs[4] = {r.a, r.b, r.c, r.d};
  const float camx = V.cam[0], camy = V.cam[1], camz = V.cam[2];
  uint32_t flags = 0u;
  TetView out;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float4 va = vs[kFacesH[f][0]], vb = vs[kFacesH[f][1]], vc = vs[kFacesH[f][2]], vo = vs[kFacesH[f][3]];
    const float e1x = fs(vc.x, va.x), e1y = fs(vc.y, va.y), e1z = fs(vc.z, va.z);
    const float e2x = fs(vb.x, va.x), e2y = fs(vb.y, va.y), e2z = fs(vb.z, va.z);
    float nx = fs(fm(e1y, e2z), fm(e1z, e2y));
    float ny = fs(fm(e1z, e2x), fm(e1x, e2z));
    float nz = fs(fm(e1x, e2y), fm(e1y, e2x));
    if (dot3x(nx, ny, nz, fs(vo.x, va.x), fs(vo.y, va.y), fs(vo.z, va.z)) < 0.0f) {
      nx = -nx; ny = -ny; nz = -nz;
      flags |= 1u << f;
    }
    out.nrm[f] = make_float4(nx, ny, nz, dot3x(nx, ny, nz, fs(va.x, camx), fs(va.y, camy), fs(va.z, camz)));
  }
  const float gx = r.b.w, gy = r.c.w, gz = r.d.w;
  const float boff = dot3x(gx, gy, gz, fs(camx, r.a.x), fs(camy, r.a.y), fs(camz, r.a.z));
  out.cb = make_float4(fa(col.x, boff), fa(col.y, boff), fa(col.z, boff), r.a.w);
  float qx[4], qy[4];
  bool behind = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float c[4];
    clip_exact(V.vp, vs[k].x, vs[k].y, vs[k].z, c);
    behind = behind || (c[3] <= 0.0f);
    const float iw = __fdividef(1.0f, c[3]);
    qx[k] = (c[0] * iw + 1.0f) * 0.5f * V.Wf;
    qy[k] = (1.0f - c[1] * iw) * 0.5f * V.Hf;
  }
  if (behind) flags |= 1u << 4;
  out.gm = make_float4(gx, gy, gz, __uint_as_float(flags));
  out.px = make_float4(qx[0], qx[1], qx[2], qx[3]);
  out.py = make_float4(qy[0], qy[1], qy[2], qy[3]);
  out.meta = make_uint4(tet, j, 0u, 0u);
  *dst = out;
}

// ---- SH colour (project_compute.wgsl:264-318) -------------------------------
constexpr float kC0 = 0.28209479177387814f, kC1 = 0.4886025119029199f;
constexpr float kC2_0 = 1.0925484305920792f, kC2_1 = -1.0925484305920792f, kC2_2 = 0.31539156525252005f,
                kC2_3 = -1.0925484305920792f, kC2_4 = 0.5462742152960396f;
constexpr float kC3_0 = -0.5900435899266435f, kC3_1 = 2.890611442640554f, kC3_2 = -0.4570457994644658f,
                kC3_3 = 0.3731763325901154f, kC3_4 = -0.4570457994644658f, kC3_5 = 1.445305721320277f,
                kC3_6 = -0.5900435899266435f;

// Coefficients are stored as fp32 training values; the shader reads them as
// f16 (crates/rmesh-viewer/src/gpu_state.rs:60-88, round to nearest even).
__device__ __forceinline__ float sh_f16(float x) { return __half2float(__float2half_rn(x)); }

// softplus with beta 10 (project_compute.wgsl:66-69)
__device__ __forceinline__ float softplus10(float x) {
  return fm(x, 10.0f) > 20.0f ? x : fm(0.1f, logf(fa(1.0f, expf(fm(10.0f, x)))));
}

// Centroid and unit direction camera -> centroid (project_compute.wgsl:268-273).
__device__ __forceinline__ float sh_direction(const TetRec& r, const float* cam, float3& centroid, float3& dir) {
  centroid = make_float3(fm(fa(fa(fa(r.a.x, r.b.x), r.c.x), r.d.x), 0.25f),
                         fm(fa(fa(fa(r.a.y, r.b.y), r.c.y), r.d.y), 0.25f),
                         fm(fa(fa(fa(r.a.z, r.b.z), r.c.z), r.d.z), 0.25f));
  const float rx = fs(centroid.x, cam[0]), ry = fs(centroid.y, cam[1]), rz = fs(centroid.z, cam[2]);
  const float len = __fsqrt_rn(dot3x(rx, ry, rz, rx, ry, rz));
  dir = len > 0.0f ? make_float3(fdv(rx, len), fdv(ry, len), fdv(rz, len)) : make_float3(0.f, 0.f, 0.f);
  return len;
}

// Colour of tet (record r, coefficients q = [3][nc] fp32) seen from cam:
// softplus(SH(dir) + 0.5 + dot(g, v0 - centroid)), evaluated term by term in
// the shader's order with explicitly rounded arithmetic.
template <int DEG>
__device__ __forceinline__ float4 sh_color(const TetRec& r, const float* __restrict__ q_in, const float* cam) {
  constexpr int NC = (DEG + 1) * (DEG + 1);
  // the tet's 3 x nc coefficients in registers; 16-byte loads when a tet's
  // row (3 nc floats) keeps 16-byte alignment (degrees 1 and 3)
  float q[3 * NC];
  if ((3 * NC) % 4 == 0) {
    const float4* q4 = reinterpret_cast<const float4*>(q_in);
#pragma unroll
    for (int i = 0; i < 3 * NC / 4; ++i) {
      const float4 v = __ldg(q4 + i);
      q[4 * i] = v.x; q[4 * i + 1] = v.y; q[4 * i + 2] = v.z; q[4 * i + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3 * NC; ++i) q[i] = __ldg(q_in + i);
  }
  float3 cen, dir;
  sh_direction(r, cam, cen, dir);
  const float x = dir.x, y = dir.y, z = dir.z;
  const float xx = fm(x, x), yy = fm(y, y), zz = fm(z, z);
  float rgb[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float* qc = q + c * NC;
    float val = fm(kC0, sh_f16(qc[0]));
    if (DEG >= 1) {
      val = fs(val, fm(fm(kC1, y), sh_f16(qc[1])));
      val = fa(val, fm(fm(kC1, z), sh_f16(qc[2])));
      val = fs(val, fm(fm(kC1, x), sh_f16(qc[3])));
    }
    if (DEG >= 2) {
      val = fa(val, fm(fm(kC2_0, fm(x, y)), sh_f16(qc[4])));
      val = fa(val, fm(fm(kC2_1, fm(y, z)), sh_f16(qc[5])));
      val = fa(val, fm(fm(kC2_2, fs(fs(fm(2.0f, zz), xx), yy)), sh_f16(qc[6])));
      val = fa(val, fm(fm(kC2_3, fm(x, z)), sh_f16(qc[7])));
      val = fa(val, fm(fm(kC2_4, fs(xx, yy)), sh_f16(qc[8])));
    }
    if (DEG >= 3) {
      val = fa(val, fm(fm(fm(kC3_0, y), fs(fm(3.0f, xx), yy)), sh_f16(qc[9])));
      val = fa(val, fm(fm(fm(fm(kC3_1, x), y), z), sh_f16(qc[10])));
      val = fa(val, fm(fm(fm(kC3_2, y), fs(fs(fm(4.0f, zz), xx), yy)), sh_f16(qc[11])));
      val = fa(val, fm(fm(fm(kC3_3, z), fs(fs(fm(2.0f, zz), fm(3.0f, xx)), fm(3.0f, yy))), sh_f16(qc[12])));
      val = fa(val, fm(fm(fm(kC3_4, x), fs(fs(fm(4.0f, zz), xx), yy)), sh_f16(qc[13])));
      val = fa(val, fm(fm(fm(kC3_5, z), fs(xx, yy)), sh_f16(qc[14])));
      val = fa(val, fm(fm(fm(kC3_6, x), fs(xx, fm(3.0f, yy))), sh_f16(qc[15])));
    }
    rgb[c] = fa(val, 0.5f);
  }
  const float off = dot3x(r.b.w, r.c.w, r.d.w, fs(r.a.x, cen.x), fs(r.a.y, cen.y), fs(r.a.z, cen.z));
  return make_float4(softplus10(fa(rgb[0], off)), softplus10(fa(rgb[1], off)), softplus10(fa(rgb[2], off)), 0.0f);
}

__device__ __forceinline__ float4 sh_color_deg(int deg, const TetRec& r, const float* q, const float* cam) {
  switch (deg) {
    case 0: return sh_color<0>(r, q, cam);
    case 1: return sh_color<1>(r, q, cam);
    case 2: return sh_color<2>(r, q, cam);
    default: return sh_color<3>(r, q, cam);
  }
}

struct ProjectArgs {
  int M;
  int n_views;
  const ViewParams* views;
  const TetRec* rec;
  // per-item outputs at the item index i = tet * n_views + view (an entry's
  // index is its item index; items that touch no tile write only vis_cnt)
  uint32_t* vis_cnt;            // tiles_touched of a tile-touching item, 0 otherwise
  float4* vis_proj;             // 2 per entry: division-projected pixel coords (emission)
  TetView* vis_view;            // per entry: the tile kernel's per-(view, tet) record
  const float4* color4;         // tet colours, [view * color_view_stride + tet]
  uint32_t color_view_stride;
  // SH colours (sh != nullptr): coefficients [M][3][nc]; the colour of each
  // tile-touching entry goes to vis_color[i]
  const float* sh;
  int sh_degree;
  float4* vis_color;
};

// One thread per (tet, view) item, items tet-major: a tet's views are
// neighbouring threads, so its record and SH coefficients are read once for
// all views.  A pure map (no scan, no block barrier): the entry data goes to
// the item's own index, and compact_keys_kernel then packs the sort keys of
// the tile-touching items in item order.
// 3 resident blocks per SM: the register cap keeps the SH coefficients of
// the 16-byte loads in registers without dropping to 2 blocks
__global__ void __launch_bounds__(256, 3) project_kernel(ProjectArgs a) {
  const unsigned long long total_items = (unsigned long long)a.M * (unsigned long long)a.n_views;
  const unsigned long long i = (unsigned long long)blockIdx.x * 256ull + threadIdx.x;
  if (i >= total_items) return;
  const uint32_t tet = (uint32_t)(i / (unsigned long long)a.n_views);
  const uint32_t view = (uint32_t)(i - (unsigned long long)tet * a.n_views);
  const ViewParams& V = a.views[view];
  const TetRec r = a.rec[tet];
  const float vx[4] = {r.a.x, r.b.x, r.c.x, r.d.x};
  const float vy[4] = {r.a.y, r.b.y, r.c.y, r.d.y};
  const float vz[4] = {r.a.z, r.b.z, r.c.z, r.d.z};
  float p[4][4], c[4][4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    clip_exact(V.vp, vx[k], vy[k], vz[k], c[k]);
    const float inv_w = fdv(1.0f, fa(c[k][3], 1e-6f));
    p[k][0] = fm(c[k][0], inv_w);
    p[k][1] = fm(c[k][1], inv_w);
    p[k][2] = fm(c[k][2], inv_w);
    p[k][3] = c[k][3];
  }
  const bool any_behind = (p[0][3] <= 0.0f) || (p[1][3] <= 0.0f) || (p[2][3] <= 0.0f) || (p[3][3] <= 0.0f);
  bool visible = true;
  if (!any_behind) {
    const float min_x = fminf(fminf(p[0][0], p[1][0]), fminf(p[2][0], p[3][0]));
    const float max_x = fmaxf(fmaxf(p[0][0], p[1][0]), fmaxf(p[2][0], p[3][0]));
    const float min_y = fminf(fminf(p[0][1], p[1][1]), fminf(p[2][1], p[3][1]));
    const float max_y = fmaxf(fmaxf(p[0][1], p[1][1]), fmaxf(p[2][1], p[3][1]));
    const float min_z = fminf(fminf(p[0][2], p[1][2]), fminf(p[2][2], p[3][2]));
    if (max_x < -1.0f || min_x > 1.0f || max_y < -1.0f || min_y > 1.0f || min_z > 1.0f) visible = false;
    const float ext_x = fm(fs(max_x, min_x), V.Wf);
    const float ext_y = fm(fs(max_y, min_y), V.Hf);
    if (fm(ext_x, ext_y) < 1.0f) visible = false;
  }
  if (visible) {  // optical-depth cull (project_compute.wgsl:146-162)
    float e2[6];
    const int ei[6] = {1, 2, 3, 2, 3, 3};
    const int ej[6] = {0, 0, 0, 1, 1, 2};
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const float dx = fs(vx[ei[e]], vx[ej[e]]), dy = fs(vy[ei[e]], vy[ej[e]]), dz = fs(vz[ei[e]], vz[ej[e]]);
      e2[e] = dot3x(dx, dy, dz, dx, dy, dz);
    }
    const float m = fmaxf(fmaxf(e2[0], fmaxf(e2[1], e2[2])), fmaxf(e2[3], fmaxf(e2[4], e2[5])));
    if (fm(r.a.w, __fsqrt_rn(m)) < 0.01f) visible = false;
  }
  uint32_t count = 0;
  if (visible && !any_behind) {
    float px[4], py[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      px[k] = fm(fm(fa(p[k][0], 1.0f), 0.5f), V.Wf);
      py[k] = fm(fm(fs(1.0f, p[k][1]), 0.5f), V.Hf);
    }
    scanline_tiles(px, py, V.Wf, V.Hf, (uint32_t)V.TS,
                   [&](uint32_t, uint32_t tx0, uint32_t tx1) { count += tx1 - tx0 + 1u; });
  }
  const bool flag = visible && count > 0u;
  a.vis_cnt[i] = flag ? count : 0u;
  if (!flag) return;
  // division-projected coords used by the emission stage (tile_gen_scan_compute.wgsl:108-117)
  float qx[4], qy[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float w = fa(c[k][3], 1e-6f);
    qx[k] = fm(fm(fa(fdv(c[k][0], w), 1.0f), 0.5f), V.Wf);
    qy[k] = fm(fm(fs(1.0f, fdv(c[k][1], w)), 0.5f), V.Hf);
  }
  a.vis_proj[2 * i] = make_float4(qx[0], qy[0], qx[1], qy[1]);
  a.vis_proj[2 * i + 1] = make_float4(qx[2], qy[2], qx[3], qy[3]);
  if (a.vis_view) {
    float4 col;
    if (a.sh) {
      const int nc = (a.sh_degree + 1) * (a.sh_degree + 1);
      col = sh_color_deg(a.sh_degree, r, a.sh + (size_t)tet * 3 * nc, V.cam);
      a.vis_color[i] = col;
    } else {
      col = a.color4[(size_t)a.color_view_stride * view + tet];
    }
    write_tet_view(a.vis_view + i, r, col, V, tet, (uint32_t)i);
  }
}

// Depth key of (tet, view) (tile_gen_scan_compute.wgsl:136-143): ~bits of the
// squared distance camera -> circumcentre minus the squared circumradius, so
// an ascending sort is back to front.
__device__ __forceinline__ uint32_t depth_key(const float4 C, const float* cam) {
  const float dx = fs(C.x, cam[0]), dy = fs(C.y, cam[1]), dz = fs(C.z, cam[2]);
  const float depth = fs(dot3x(dx, dy, dz, dx, dy, dz), C.w);
  return ~__float_as_uint(depth);
}

// Sort keys of the tile-touching items, compacted in item order (within one
// view: ascending tet id, the tie order of the stable depth sort):
//   key = count << 40 | view << 32 | ~bits(depth),  value = item index.
// The sort orders bits 0..31 only; the view (< 64) in bits 32..39 and the tile
// count in bits 40..63 ride along for the emission stage (the count saturated
// at kKeyCountMax, which then reads vis_cnt).  A chained scan over blocks of kCompactItems items, each thread
// taking kCompactPerThread consecutive items.
constexpr int kCompactPerThread = 8;
constexpr int kCompactItems = 256 * kCompactPerThread;
constexpr uint32_t kKeyCountMax = (1u << 24) - 1u;

struct CompactArgs {
  int M;
  int n_views;
  const ViewParams* views;
  const float4* circ;
  const uint32_t* vis_cnt;
  unsigned long long* vis_key;
  uint32_t* vis_val;
  unsigned long long* status;  // chained-scan status, one word per block (zeroed)
  uint32_t* ticket;            // block ticket (zeroed)
  Counters* counters;
};

__global__ void __launch_bounds__(256) compact_keys_kernel(CompactArgs a) {
  __shared__ uint32_t s_blk;
  __shared__ uint32_t s_warp[8];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_blk = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const uint32_t blk = s_blk;
  const unsigned long long total_items = (unsigned long long)a.M * (unsigned long long)a.n_views;
  const unsigned long long i0 = (unsigned long long)blk * kCompactItems + (unsigned long long)threadIdx.x * kCompactPerThread;
  uint32_t cnt[kCompactPerThread];
  if (i0 + kCompactPerThread <= total_items) {  // i0 is a multiple of 8: 32-byte aligned
    const uint4 c0 = __ldg(reinterpret_cast<const uint4*>(a.vis_cnt + i0));
    const uint4 c1 = __ldg(reinterpret_cast<const uint4*>(a.vis_cnt + i0 + 4));
    cnt[0] = c0.x; cnt[1] = c0.y; cnt[2] = c0.z; cnt[3] = c0.w;
    cnt[4] = c1.x; cnt[5] = c1.y; cnt[6] = c1.z; cnt[7] = c1.w;
  } else {
#pragma unroll
    for (int q = 0; q < kCompactPerThread; ++q) cnt[q] = i0 + q < total_items ? a.vis_cnt[i0 + q] : 0u;
  }
  uint32_t mine = 0;
#pragma unroll
  for (int q = 0; q < kCompactPerThread; ++q) mine += cnt[q] ? 1u : 0u;
  // block exclusive scan of the per-thread flag counts
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t warp_off = 0, block_total = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const uint32_t c = s_warp[w];
    if (w < warp) warp_off += c;
    block_total += c;
  }
  if (warp == 0) {
    const unsigned long long pre = chained_lookback(a.status, blk, block_total, &a.counters->err);
    if (lane == 0) s_prefix = pre;
  }
  __syncthreads();
  unsigned long long j = s_prefix + warp_off + x - mine;
  if (mine) {
    uint32_t tet = (uint32_t)(i0 / (unsigned long long)a.n_views);
    uint32_t view = (uint32_t)(i0 - (unsigned long long)tet * a.n_views);
    float4 C = a.circ[tet];
#pragma unroll
    for (int q = 0; q < kCompactPerThread; ++q) {
      if (cnt[q]) {
        const unsigned long long c24 = cnt[q] < kKeyCountMax ? cnt[q] : kKeyCountMax;
        a.vis_key[j] = (c24 << 40) | ((unsigned long long)view << 32) | depth_key(C, a.views[view].cam);
        a.vis_val[j] = (uint32_t)(i0 + q);
        ++j;
      }
      if (++view == (uint32_t)a.n_views && q + 1 < kCompactPerThread) {
        view = 0;
        ++tet;
        if (i0 + q + 1 < total_items) C = a.circ[tet];
      }
    }
  }
  // the block holding the last item publishes the compacted count
  if (threadIdx.x == 0 && (unsigned long long)(blk + 1) * kCompactItems >= total_items &&
      (unsigned long long)blk * kCompactItems < total_items)
    a.counters->n_vis = (uint32_t)(s_prefix + block_total);
}

}  // namespace rm
