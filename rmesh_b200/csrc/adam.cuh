// Gradient gather and fused multi-group Adam.
//
// The adjoint accumulates, per tet, a 20-float slot: [0] density, [1..3] base
// colour, [4..6] colour gradient, [7..18] the four vertices' xyz.  Vertex
// gradients are then gathered through a CSR map vertex -> (tet*4 + corner)
// built once per topology, so no vertex-level atomics are needed.
//
// Adam restates crates/rmesh-train/src/wgsl/adam_compute.wgsl:121-149 per
// element (NaN -> 0, clip to +-1e20, bias correction exp(step*ln(beta)),
// safe_div / safe_sqrt), for every group in ONE launch: vertices (lr_verts),
// densities (lr_dens), colour gradients (lr_grads), base colours when
// lr_base > 0 (the reference's train_step leaves base colours untouched,
// crates/rmesh-python/src/lib.rs:393-439, 2590-2626), and SH coefficients
// (lr_sh) when the mesh is coloured by spherical harmonics.  The step is skipped
// entirely when the run raised an error (e.g. pair overflow), so the host can
// grow its buffers and redo the step.
#pragma once
#include "common.cuh"

namespace rm {

__device__ __forceinline__ void adam_elem(float& p, float& m, float& v, float g_raw, float lr, float b1, float b2,
                                          float eps, float b1p, float b2p) {
  const float g = clipf(g_raw != g_raw ? 0.0f : g_raw, kMinVal, kMaxVal);
  const float m_new = __fadd_rn(__fmul_rn(b1, m), __fmul_rn(__fsub_rn(1.0f, b1), g));
  m = m_new;
  const float v_new = __fadd_rn(__fmul_rn(b2, v), __fmul_rn(__fmul_rn(__fsub_rn(1.0f, b2), g), g));
  v = v_new;
  const float m_hat = safe_div(m_new, __fsub_rn(1.0f, b1p));
  const float v_hat = safe_div(v_new, __fsub_rn(1.0f, b2p));
  p = __fsub_rn(p, __fmul_rn(lr, safe_div(m_hat, __fadd_rn(safe_sqrt(v_hat), eps))));
}

__device__ __forceinline__ float gather_vertex_grad(const float* __restrict__ slot, const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ ref, uint32_t vtx, int c) {
  float s = 0.0f;
  for (uint32_t i = off[vtx]; i < off[vtx + 1]; ++i) {
    const uint32_t r = ref[i];
    s += slot[(size_t)(r >> 2) * kGradSlot + 7 + (r & 3u) * 3 + c];
  }
  return s;
}

struct AdamArgs {
  int N, M;
  float* verts;
  float* dens;
  float* cgrad;
  float* base;
  float* m_verts; float* v_verts;
  float* m_dens; float* v_dens;
  float* m_cgrad; float* v_cgrad;
  float* m_base; float* v_base;
  const float* grad_slot;
  float* sh; float* m_sh; float* v_sh;  // SH coefficients (nullptr: base colours)
  const float* d_sh;
  long long n_sh;
  const uint32_t* csr_off;
  const uint32_t* csr_ref;
  const AdamParams* hp;
  const Counters* counters;
  int n_counters;            // number of Counters blocks to check for errors
};

__global__ void __launch_bounds__(256) adam_kernel(AdamArgs a) {
  for (int c = 0; c < a.n_counters; ++c)
    if (a.counters[c].err) return;
  const AdamParams hp = *a.hp;
  const float step_f = (float)hp.step;
  const float b1p = expf(step_f * logf(hp.beta1));
  const float b2p = expf(step_f * logf(hp.beta2));
  // units: N vertices, M tets, then the SH coefficients four at a time (16-byte
  // loads and stores: the coefficient arrays and their gradients start on
  // 16-byte boundaries), the last unit taking the 1-3 left over one by one
  const long long n_sh = a.sh && hp.lr_sh > 0.0f ? a.n_sh : 0;
  const long long total = (long long)a.N + a.M + (n_sh + 3) / 4;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    if (i >= (long long)a.N + a.M) {
      const long long e0 = 4 * (i - a.N - a.M);
      if (e0 + 4 <= n_sh) {
        const size_t q = (size_t)(e0 >> 2);
        float4 p = reinterpret_cast<float4*>(a.sh)[q];
        float4 m = reinterpret_cast<float4*>(a.m_sh)[q];
        float4 v = reinterpret_cast<float4*>(a.v_sh)[q];
        const float4 g = reinterpret_cast<const float4*>(a.d_sh)[q];
        adam_elem(p.x, m.x, v.x, g.x, hp.lr_sh, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
        adam_elem(p.y, m.y, v.y, g.y, hp.lr_sh, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
        adam_elem(p.z, m.z, v.z, g.z, hp.lr_sh, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
        adam_elem(p.w, m.w, v.w, g.w, hp.lr_sh, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
        reinterpret_cast<float4*>(a.sh)[q] = p;
        reinterpret_cast<float4*>(a.m_sh)[q] = m;
        reinterpret_cast<float4*>(a.v_sh)[q] = v;
      } else {
        for (long long e = e0; e < n_sh; ++e)
          adam_elem(a.sh[e], a.m_sh[e], a.v_sh[e], a.d_sh[e], hp.lr_sh, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
      }
    } else if (i < a.N) {
      const uint32_t vtx = (uint32_t)i;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float g = gather_vertex_grad(a.grad_slot, a.csr_off, a.csr_ref, vtx, c);
        const size_t e = 3 * (size_t)vtx + c;
        adam_elem(a.verts[e], a.m_verts[e], a.v_verts[e], g, hp.lr_verts, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
      }
    } else {
      const size_t t = (size_t)(i - a.N);
      const float* sl = a.grad_slot + t * kGradSlot;
      adam_elem(a.dens[t], a.m_dens[t], a.v_dens[t], sl[0], hp.lr_dens, hp.beta1, hp.beta2, hp.eps, b1p, b2p);
#pragma unroll
      for (int c = 0; c < 3; ++c)
        adam_elem(a.cgrad[3 * t + c], a.m_cgrad[3 * t + c], a.v_cgrad[3 * t + c], sl[4 + c], hp.lr_grads, hp.beta1,
                  hp.beta2, hp.eps, b1p, b2p);
      if (hp.lr_base > 0.0f) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          adam_elem(a.base[3 * t + c], a.m_base[3 * t + c], a.v_base[3 * t + c], sl[1 + c], hp.lr_base, hp.beta1,
                    hp.beta2, hp.eps, b1p, b2p);
      }
    }
  }
}

// Unpack slots into the reference's gradient arrays (backward() API):
// d_vertices[3N], d_densities[M], d_base_colors[3M], d_color_grads[3M].
__global__ void __launch_bounds__(256) unpack_grads_kernel(int N, int M, const float* __restrict__ slot,
                                                           const uint32_t* __restrict__ csr_off,
                                                           const uint32_t* __restrict__ csr_ref, float* d_verts,
                                                           float* d_dens, float* d_base, float* d_cgrad) {
  const long long total = (long long)N + M;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    if (i < N) {
      for (int c = 0; c < 3; ++c) d_verts[3 * i + c] = gather_vertex_grad(slot, csr_off, csr_ref, (uint32_t)i, c);
    } else {
      const size_t t = (size_t)(i - N);
      const float* sl = slot + t * kGradSlot;
      d_dens[t] = sl[0];
      for (int c = 0; c < 3; ++c) {
        d_base[3 * t + c] = sl[1 + c];
        d_cgrad[3 * t + c] = sl[4 + c];
      }
    }
  }
}

// CSR construction helpers: refs (tet*4 + corner) are radix-sorted by vertex id
// on the device; offsets are then found from the sorted vertex keys.
__global__ void csr_fill_kernel(int M, const uint32_t* __restrict__ idx, uint32_t* keys, uint32_t* refs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 4ll * M) return;
  keys[i] = idx[i];
  refs[i] = (uint32_t)i;
}

__global__ void csr_offsets_kernel(int n_refs, int N, const uint32_t* __restrict__ sorted_keys, uint32_t* off) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n_refs) return;
  // off[v] = first i with key >= v
  const uint32_t cur = i < n_refs ? sorted_keys[i] : (uint32_t)N;
  const uint32_t prev = i > 0 ? sorted_keys[i - 1] : 0u;
  const uint32_t lo = i > 0 ? prev + 1u : 0u;
  for (uint32_t v = lo; v <= cur && v <= (uint32_t)N; ++v) off[v] = (uint32_t)i;
}

}  // namespace rm
