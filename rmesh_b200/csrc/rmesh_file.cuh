// Device decode of a .rmesh scene (crates/rmesh-data/src/lib.rs:247-393).
//
// The host parses the header and slices the file into its sections; these
// kernels turn the packed sections into the renderer's fp32 buffers:
//   densities    exp((u8 - 100) / 20), through a 256-entry table the host
//                fills with the same float expf the reference's loader uses
//   colour grads f16 -> f32
//   SH           PCA decompression, coeff[t][f] = mean[f] + sum_k w[t][k] *
//                basis[k][f], accumulated in f32 in k order with separately
//                rounded multiplies and adds (the loader's loop, lib.rs:350-359)
//   circumdata   circumsphere in double with the loader's degenerate-tet rules
//                (lib.rs:601-707), explicitly rounded so no FMA is contracted
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"

namespace rm {

struct DensityTable {
  float v[256];
};

__device__ __forceinline__ float half_bits(uint16_t h) { return __half2float(__ushort_as_half(h)); }

struct DVec {
  double x, y, z;
};
__device__ __forceinline__ DVec dv(double x, double y, double z) { return DVec{x, y, z}; }
__device__ __forceinline__ DVec dsub(DVec a, DVec b) {
  return dv(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z));
}
__device__ __forceinline__ DVec dadd(DVec a, DVec b) {
  return dv(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z));
}
__device__ __forceinline__ DVec dscale(DVec a, double s) {
  return dv(__dmul_rn(a.x, s), __dmul_rn(a.y, s), __dmul_rn(a.z, s));
}
__device__ __forceinline__ double ddot(DVec a, DVec b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
// (a.y b.z - b.y a.z, a.z b.x - b.z a.x, a.x b.y - b.x a.y)
__device__ __forceinline__ DVec dcross(DVec a, DVec b) {
  return dv(__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(b.y, a.z)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(b.z, a.x)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(b.x, a.y)));
}
__device__ __forceinline__ double dlen(DVec a) { return __dsqrt_rn(ddot(a, a)); }

__device__ __forceinline__ float4 circumsphere_f64(const float* __restrict__ verts, const uint32_t* q) {
  DVec v[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    v[k] = dv((double)verts[3 * (size_t)q[k]], (double)verts[3 * (size_t)q[k] + 1], (double)verts[3 * (size_t)q[k] + 2]);
  const DVec a = dsub(v[1], v[0]), b = dsub(v[2], v[0]), c = dsub(v[3], v[0]);
  const double aa = ddot(a, a), bb = ddot(b, b), cc = ddot(c, c);
  const DVec bc = dcross(b, c), ca = dcross(c, a), ab = dcross(a, b);
  const double denom = __dmul_rn(2.0, ddot(a, bc));
  if (fabs(denom) < 1e-10) {
    double md = dlen(dsub(v[1], v[0]));
    md = fmax(md, dlen(dsub(v[2], v[0])));
    md = fmax(md, dlen(dsub(v[3], v[0])));
    md = fmax(md, dlen(dsub(v[2], v[1])));
    md = fmax(md, dlen(dsub(v[3], v[1])));
    md = fmax(md, dlen(dsub(v[3], v[2])));
    const DVec cen = dscale(dadd(dadd(dadd(v[0], v[1]), v[2]), v[3]), 0.25);
    float r2 = 1e20f;  // near-planar: sorts to the back
    if (md < 1e-7) {
      double r = dlen(dsub(v[0], cen));
      r = fmin(r, dlen(dsub(v[1], cen)));
      r = fmin(r, dlen(dsub(v[2], cen)));
      r = fmin(r, dlen(dsub(v[3], cen)));
      r2 = (float)__dmul_rn(r, r);
    }
    return make_float4((float)cen.x, (float)cen.y, (float)cen.z, r2);
  }
  const DVec num = dadd(dadd(dscale(bc, aa), dscale(ca, bb)), dscale(ab, cc));
  const DVec rel = dv(__ddiv_rn(num.x, denom), __ddiv_rn(num.y, denom), __ddiv_rn(num.z, denom));
  const DVec cen = dadd(v[0], rel);
  return make_float4((float)cen.x, (float)cen.y, (float)cen.z, (float)ddot(rel, rel));
}

struct SceneDecodeArgs {
  uint64_t M;
  uint32_t D, K;  // SH features per tet (3 nc), PCA components used
  const float* verts;
  const uint32_t* idx;
  const uint8_t* log_dens;
  const uint16_t* mean;     // [D] f16
  const uint16_t* basis;    // [K][D] f16
  const uint16_t* weights;  // [M][K] f16
  const uint16_t* grads16;  // [3M] f16 or nullptr
  float* dens;
  float* grads;
  float* sh;
  float4* circ;
  DensityTable table;
};

// one thread per tet: density, colour gradient, circumsphere
__global__ void __launch_bounds__(256) decode_tets_kernel(SceneDecodeArgs a) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < a.M; t += (uint64_t)gridDim.x * blockDim.x) {
    a.dens[t] = a.table.v[a.log_dens[t]];
#pragma unroll
    for (int c = 0; c < 3; ++c) a.grads[3 * t + c] = a.grads16 ? half_bits(a.grads16[3 * t + c]) : 0.0f;
    a.circ[t] = circumsphere_f64(a.verts, a.idx + 4 * t);
  }
}

// one thread per (tet, SH feature): PCA decompression
__global__ void __launch_bounds__(256) pca_decode_kernel(SceneDecodeArgs a) {
  const uint64_t total = a.M * a.D;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t t = i / a.D;
    const uint32_t f = (uint32_t)(i - t * a.D);
    float val = half_bits(a.mean[f]);
    const uint16_t* w = a.weights + t * a.K;
    for (uint32_t q = 0; q < a.K; ++q) val = __fadd_rn(val, __fmul_rn(half_bits(w[q]), half_bits(a.basis[(size_t)q * a.D + f])));
    a.sh[i] = val;
  }
}

}  // namespace rm
