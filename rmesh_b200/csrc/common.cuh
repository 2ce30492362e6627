// Shared device definitions for the B200 rmeshvk tiled path.
//
// Exactness: the per-tet stages whose integer outputs must match the reference
// bit for bit (tile counts, tile enumeration, depth keys, row spans) use the
// explicitly rounded intrinsics below, so nvcc can neither contract a multiply
// and add into an FMA nor swap the order of the left-to-right WGSL evaluation
// (crates/rmesh-render/src/wgsl/project_compute.wgsl:113-262,
//  crates/rmesh-tile/src/wgsl/tile_gen_scan_compute.wgsl:96-201).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rm {

constexpr int kMaxViews = 64;
constexpr uint32_t kSentinel = 0xFFFFFFFFu;
constexpr int kGradSlot = 20;  // floats per tet gradient slot (19 used, 16-byte multiple)

// Device status bits (also returned through the C ABI).
enum : uint32_t {
  kErrPairOverflow = 1u << 0,   // more (tile, tet) pairs than the pair buffers hold
  kErrSpinTimeout = 1u << 1,    // a bounded spin (look-back / mbarrier) gave up
};

// Per-view constants, device resident, refreshed every call from pinned host memory.
struct ViewParams {
  float vp[16];      // column-major view-projection
  float c2w[9];      // column-major camera-to-world rotation
  float fx, fy, cx, cy;
  float cam[3];
  float min_t;
  float Wf, Hf;      // width/height as float (the reference's uniforms.screen_width)
  float n_pixels;    // f32(W*H), the loss normaliser (loss_compute.wgsl:34)
  int W, H, TS;
  int tiles_x, tiles_y;
  uint32_t tile_base;  // first global tile id of this view
  uint32_t pix_base;   // first pixel of this view in the concatenated image arrays
  uint32_t pad[2];
};

// Device counters of one pipeline run (zeroed by a memset before each run).
struct Counters {
  uint32_t n_vis;                  // visible (tile-touching) tets over all views
  uint32_t err;                    // kErr* bits
  unsigned long long n_pairs;      // total (tile, tet) slots over all views
  uint32_t tile_ticket;            // persistent tile-queue head
  uint32_t pad0;
  uint32_t shortfall[kMaxViews];   // view emitted fewer pairs than it counted
  double loss[kMaxViews];          // per-view loss value (sum over RGB and pixels / n_pixels)
};

// Training hyper-parameters, device resident (so a captured graph picks up new values).
struct AdamParams {
  uint32_t step;
  float lr_verts, lr_dens, lr_grads, lr_base, lr_sh;
  float beta1, beta2, eps;
  int loss_type;  // 0 = L1, 1 = L2
};

// ---- explicitly rounded arithmetic (no contraction) ----------------------
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float dot3x(float ax, float ay, float az, float bx, float by, float bz) {
  return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

// clip = vp * vec4(x, y, z, 1): ((c0*x + c1*y) + c2*z) + c3 per row.
__device__ __forceinline__ void clip_exact(const float* vp, float x, float y, float z, float c[4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r) c[r] = fa(fa(fa(fm(vp[r], x), fm(vp[4 + r], y)), fm(vp[8 + r], z)), vp[12 + r]);
}

// ---- safe math (crates/rmesh-util/src/wgsl/math.wgsl:3-65) ----------------
constexpr float kTiny = 1.0754944e-20f;
constexpr float kMinVal = -1e+20f;
constexpr float kMaxVal = 1e+20f;
constexpr float kLogMax = 46.0517f;

__device__ __forceinline__ float clipf(float v, float lo, float hi) { return fmaxf(fminf(v, hi), lo); }
__device__ __forceinline__ float safe_div(float a, float b) {
  return fabsf(b) < kTiny ? clipf(a / kTiny, kMinVal, kMaxVal) : clipf(a / b, kMinVal, kMaxVal);
}
__device__ __forceinline__ float safe_exp(float v) { return expf(clipf(v, -88.0f, kLogMax)); }
__device__ __forceinline__ float safe_sqrt(float a) { return a < kTiny ? 0.0f : sqrtf(a); }
__device__ __forceinline__ float phi_f(float x) {
  if (fabsf(x) < 0.02f) return 1.0f + x * (-0.5f + x * (1.0f / 6.0f + x * (-1.0f / 24.0f)));
  return safe_div(1.0f - expf(-x), x);
}
__device__ __forceinline__ float dphi_f(float x) {
  if (fabsf(x) < 0.02f) return -0.5f + x * (1.0f / 3.0f + x * (-1.0f / 8.0f + x * (1.0f / 30.0f)));
  float ex = expf(-x);
  return safe_div(ex * (x + 1.0f) - 1.0f, x * x);
}

// FACES (crates/rmesh-util/src/wgsl/intersect.wgsl:4-10): (a, b, c, opposite).
__constant__ int8_t kFaces[4][4] = {{0, 2, 1, 3}, {1, 2, 3, 0}, {0, 3, 2, 1}, {3, 0, 1, 2}};
// the same table for compile-time-unrolled loops
__device__ constexpr int kFacesH[4][4] = {{0, 2, 1, 3}, {1, 2, 3, 0}, {0, 3, 2, 1}, {3, 0, 1, 2}};

// ---- bounded spin helpers --------------------------------------------------
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
  *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Chained-scan status word: [63:62] flag (1 aggregate, 2 inclusive), [61:0] value.
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1ull;

// Decoupled look-back over earlier blocks (single-pass chained scan).  Called by
// warp 0 of a block whose position in the scan is `blk` (taken from a ticket so
// earlier positions were started first).  Publishes `total`, returns the
// exclusive prefix to every lane of warp 0.  Spins are bounded: on timeout the
// missing predecessor counts as 0 and kErrSpinTimeout is raised.
__device__ __forceinline__ unsigned long long chained_lookback(unsigned long long* status, uint32_t blk,
                                                               unsigned long long total, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  if (blk == 0) {
    if (lane == 0) {
      __threadfence();
      st_volatile_u64(&status[0], kFlagInc | total);
    }
    return 0ull;
  }
  if (lane == 0) {
    __threadfence();
    st_volatile_u64(&status[blk], kFlagAgg | total);
  }
  unsigned long long prefix = 0ull;
  int64_t base = (int64_t)blk - 1;
  uint32_t spins = 0;
  bool timed_out = false;
  while (true) {
    int64_t p = base - lane;
    unsigned long long s = (p >= 0) ? ld_volatile_u64(&status[p]) : kFlagInc;  // p < 0: virtual zero
    // Wait until every lane sees a published word (or a virtual inclusive one).
    while (__any_sync(0xffffffffu, (s >> 62) == 0ull)) {
      if (++spins > kSpinLimit) { timed_out = true; break; }
      __nanosleep(32);
      if ((s >> 62) == 0ull) s = ld_volatile_u64(&status[p]);
    }
    if (timed_out) {
      if ((s >> 62) == 0ull) s = kFlagInc;  // treat missing as zero, stop here
    }
    unsigned inc_mask = __ballot_sync(0xffffffffu, (s >> 62) == 2ull);
    unsigned long long v = s & kValMask;
    if (inc_mask) {
      int first = __ffs(inc_mask) - 1;  // nearest inclusive predecessor
      if (lane > first) v = 0ull;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      prefix += v;
      break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    prefix += v;
    base -= 32;
  }
  if (lane == 0) {
    if (timed_out) atomicOr(err, kErrSpinTimeout);
    __threadfence();
    st_volatile_u64(&status[blk], kFlagInc | ((prefix + total) & kValMask));
  }
  return prefix;
}

// View lookup by global tile id (views are stored in tile order).
__device__ __forceinline__ int view_of_tile(const ViewParams* views, int n_views, uint32_t tile) {
  int lo = 0, hi = n_views - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (views[mid].tile_base <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

}  // namespace rm
