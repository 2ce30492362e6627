// Adjoint of the spherical-harmonics colour.
//
// The forward colour is the reference's (project_compute.wgsl:264-318, restated
// in sh_color): per view, colour = softplus(SH(dir) + 0.5 + dot(g, v0 - c)) with
// c the tet centroid and dir = normalize(c - cam).  The reference has no
// adjoint for it; this kernel is one.  The tile kernel leaves, for every
// tile-touching (view, tet) entry j, the gradient of the loss with respect to
// that entry's colour in vis_dcolor[j], j = tet * n_views + view.  One thread
// per tet then walks the run's views (an entry exists where vis_cnt[j] > 0, the
// tet touched a tile of that view; its gradients are contiguous), and chains
// the colour gradient through softplus (math.wgsl:27-33), the SH basis, the
// offset dot(g, v0 - c) and the view direction:
//   d coeff[ch][i] += d_rgb[ch] * basis_i(dir)
//   d g            += S (v0 - c),      S = sum over channels of d_rgb
//   d v0           += S g,             d c = -S g + (I - dir dir^T) d_dir / |c - cam|
//   d v_k          += d c / 4
// with d_dir = sum_ch d_rgb[ch] sum_i coeff[ch][i] grad basis_i(dir).  Each
// thread owns its tet, so the results are added to the gradient slot and the
// coefficient gradient without atomics (the tile kernel has finished).
#pragma once
#include "common.cuh"
#include "project.cuh"

namespace rm {

// basis_i(dir) and its gradient with the direction components taken as independent
template <int DEG>
__device__ __forceinline__ void sh_basis_all(float x, float y, float z, float* b, float* gx, float* gy, float* gz) {
  const float xx = x * x, yy = y * y, zz = z * z;
  b[0] = kC0; gx[0] = 0.f; gy[0] = 0.f; gz[0] = 0.f;
  if (DEG >= 1) {
    b[1] = -kC1 * y; gx[1] = 0.f; gy[1] = -kC1; gz[1] = 0.f;
    b[2] = kC1 * z;  gx[2] = 0.f; gy[2] = 0.f;  gz[2] = kC1;
    b[3] = -kC1 * x; gx[3] = -kC1; gy[3] = 0.f; gz[3] = 0.f;
  }
  if (DEG >= 2) {
    b[4] = kC2_0 * x * y; gx[4] = kC2_0 * y; gy[4] = kC2_0 * x; gz[4] = 0.f;
    b[5] = kC2_1 * y * z; gx[5] = 0.f; gy[5] = kC2_1 * z; gz[5] = kC2_1 * y;
    b[6] = kC2_2 * (2.f * zz - xx - yy); gx[6] = -2.f * kC2_2 * x; gy[6] = -2.f * kC2_2 * y; gz[6] = 4.f * kC2_2 * z;
    b[7] = kC2_3 * x * z; gx[7] = kC2_3 * z; gy[7] = 0.f; gz[7] = kC2_3 * x;
    b[8] = kC2_4 * (xx - yy); gx[8] = 2.f * kC2_4 * x; gy[8] = -2.f * kC2_4 * y; gz[8] = 0.f;
  }
  if (DEG >= 3) {
    b[9] = kC3_0 * y * (3.f * xx - yy);
    gx[9] = 6.f * kC3_0 * x * y; gy[9] = kC3_0 * (3.f * xx - 3.f * yy); gz[9] = 0.f;
    b[10] = kC3_1 * x * y * z;
    gx[10] = kC3_1 * y * z; gy[10] = kC3_1 * x * z; gz[10] = kC3_1 * x * y;
    b[11] = kC3_2 * y * (4.f * zz - xx - yy);
    gx[11] = -2.f * kC3_2 * x * y; gy[11] = kC3_2 * (4.f * zz - xx - 3.f * yy); gz[11] = 8.f * kC3_2 * y * z;
    b[12] = kC3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
    gx[12] = -6.f * kC3_3 * x * z; gy[12] = -6.f * kC3_3 * y * z; gz[12] = kC3_3 * (6.f * zz - 3.f * xx - 3.f * yy);
    b[13] = kC3_4 * x * (4.f * zz - xx - yy);
    gx[13] = kC3_4 * (4.f * zz - 3.f * xx - yy); gy[13] = -2.f * kC3_4 * x * y; gz[13] = 8.f * kC3_4 * x * z;
    b[14] = kC3_5 * z * (xx - yy);
    gx[14] = 2.f * kC3_5 * x * z; gy[14] = -2.f * kC3_5 * y * z; gz[14] = kC3_5 * (xx - yy);
    b[15] = kC3_6 * x * (xx - 3.f * yy);
    gx[15] = kC3_6 * (3.f * xx - 3.f * yy); gy[15] = -6.f * kC3_6 * x * y; gz[15] = 0.f;
  }
}

// d softplus10(x) / dx (math.wgsl:27-33)
__device__ __forceinline__ float dsoftplus10(float x) {
  if (x * 10.0f > 20.0f) return 1.0f;
  const float e = expf(10.0f * x);
  return safe_div(e, 1.0f + e);
}

struct ShBackwardArgs {
  int M;
  int n_views;
  const ViewParams* views;
  const TetRec* rec;
  const float* sh;           // [M][3][nc] fp32 coefficients (read as f16, as in the forward)
  const uint32_t* vis_cnt;   // [M * n_views] tiles touched by (tet, view) at tet * n_views + view
  const float4* vis_dcolor;  // [M * n_views] colour gradient per entry
  float* d_sh;               // [M][3][nc], accumulated
  float* grad_slot;          // [M][kGradSlot], colour gradient [4..6] and vertices [7..18] accumulated
};

// 4 resident blocks per SM (the register cap keeps the degree-3 coefficient
// and gradient arrays in registers)
template <int DEG>
__global__ void __launch_bounds__(128, 4) sh_backward_kernel(ShBackwardArgs a) {
  constexpr int NC = (DEG + 1) * (DEG + 1);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.M) return;
  bool any = false;
  for (int v = 0; v < a.n_views && !any; ++v) any = a.vis_cnt[(size_t)t * a.n_views + v] != 0u;
  if (!any) return;
  const TetRec r = a.rec[t];
  // a tet's 3 nc floats keep 16-byte alignment at degrees 1 and 3: vector
  // loads and stores there
  constexpr bool kVec = (3 * NC) % 4 == 0;
  float q[3 * NC], dq[3 * NC];
  const float* src = a.sh + (size_t)t * 3 * NC;
  if (kVec) {
#pragma unroll
    for (int i = 0; i < 3 * NC / 4; ++i) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(src) + i);
      q[4 * i] = sh_f16(v.x); q[4 * i + 1] = sh_f16(v.y); q[4 * i + 2] = sh_f16(v.z); q[4 * i + 3] = sh_f16(v.w);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3 * NC; ++i) q[i] = sh_f16(src[i]);
  }
#pragma unroll
  for (int i = 0; i < 3 * NC; ++i) dq[i] = 0.0f;
  const float gx = r.b.w, gy = r.c.w, gz = r.d.w;
  float dg0 = 0.f, dg1 = 0.f, dg2 = 0.f;
  float dc0 = 0.f, dc1 = 0.f, dc2 = 0.f;  // d centroid
  float dv00 = 0.f, dv01 = 0.f, dv02 = 0.f;  // d v0 beyond the centroid share
  for (int v = 0; v < a.n_views; ++v) {
    const size_t j = (size_t)t * a.n_views + v;
    if (a.vis_cnt[j] == 0u) continue;
    const float4 dcol = a.vis_dcolor[j];
    if (dcol.x == 0.f && dcol.y == 0.f && dcol.z == 0.f) continue;
    float3 cen, dir;
    const float len = sh_direction(r, a.views[v].cam, cen, dir);
    float b[NC], bx[NC], by[NC], bz[NC];
    sh_basis_all<DEG>(dir.x, dir.y, dir.z, b, bx, by, bz);
    const float ox = r.a.x - cen.x, oy = r.a.y - cen.y, oz = r.a.z - cen.z;
    const float off = gx * ox + gy * oy + gz * oz;
    const float dcc[3] = {dcol.x, dcol.y, dcol.z};
    float S = 0.f, ddx = 0.f, ddy = 0.f, ddz = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float val = 0.f;
#pragma unroll
      for (int i = 0; i < NC; ++i) val += b[i] * q[c * NC + i];
      const float drgb = dcc[c] * dsoftplus10(val + 0.5f + off);
      S += drgb;
#pragma unroll
      for (int i = 0; i < NC; ++i) {
        dq[c * NC + i] += drgb * b[i];
        const float w = drgb * q[c * NC + i];
        ddx += w * bx[i];
        ddy += w * by[i];
        ddz += w * bz[i];
      }
    }
    dg0 += S * ox; dg1 += S * oy; dg2 += S * oz;
    dv00 += S * gx; dv01 += S * gy; dv02 += S * gz;
    dc0 -= S * gx; dc1 -= S * gy; dc2 -= S * gz;
    if (len > 0.0f) {
      const float dd = dir.x * ddx + dir.y * ddy + dir.z * ddz;
      const float il = 1.0f / len;
      dc0 += (ddx - dir.x * dd) * il;
      dc1 += (ddy - dir.y * dd) * il;
      dc2 += (ddz - dir.z * dd) * il;
    }
  }
  float* dst = a.d_sh + (size_t)t * 3 * NC;
  if (kVec) {
#pragma unroll
    for (int i = 0; i < 3 * NC / 4; ++i) {
      float4* d4 = reinterpret_cast<float4*>(dst) + i;
      float4 v = *d4;
      v.x += dq[4 * i]; v.y += dq[4 * i + 1]; v.z += dq[4 * i + 2]; v.w += dq[4 * i + 3];
      *d4 = v;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3 * NC; ++i) dst[i] += dq[i];
  }
  float* sl = a.grad_slot + (size_t)t * kGradSlot;
  sl[4] += dg0; sl[5] += dg1; sl[6] += dg2;
  const float qx = 0.25f * dc0, qy = 0.25f * dc1, qz = 0.25f * dc2;
  sl[7] += qx + dv00; sl[8] += qy + dv01; sl[9] += qz + dv02;
#pragma unroll
  for (int k = 1; k < 4; ++k) {
    sl[7 + 3 * k] += qx;
    sl[8 + 3 * k] += qy;
    sl[9 + 3 * k] += qz;
  }
}

}  // namespace rm
