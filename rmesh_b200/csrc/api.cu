// C-ABI implementation: context, device buffers and stage sequencing.
//
// Host sequencing restates crates/rmesh-python/src/lib.rs:
//   forward_tiled  :1041-1204   backward :1894-2031   train_step :2405-2636
// with three B200 changes: (1) no host readback between stages -- counts stay
// on the device and every kernel reads them from there; (2) the adjoint reuses
// the forward's sorted tile lists instead of re-sorting; (3) train steps run the
// fused forward+loss+adjoint tile kernel and one multi-group Adam launch.
//
// Capacity: pair buffers start from an estimate; a run that overflows raises a
// device bit, Adam is skipped on the device, and the host grows the buffers to
// the exact count and repeats the call.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rmesh_b200.h"
#include "adam.cuh"
#include "bin.cuh"
#include "common.cuh"
#include "project.cuh"
#include "rmesh_file.cuh"
#include "sh.cuh"
#include "sort.cuh"
#include "tile.cuh"

using namespace rm;

static_assert(sizeof(Counters) == 792, "Counters layout is mirrored by the Python binding");

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // grows (never shrinks); returns a cudaError_t; *grew set when reallocated
  cudaError_t ensure(size_t n, bool* grew = nullptr) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    size_t want = std::max<size_t>(n, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    bytes = want;
    if (grew) *grew = true;
    return cudaSuccess;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

enum Stage { kStRecords = 0, kStProject, kStTetSort, kStEmit, kStPairSort, kStRanges, kStComposite, kStAdam, kStShAdjoint };
// NVTX range names of the stages (profilers can select kernels by them, e.g.
// ncu --nvtx --nvtx-include "rmesh/composite/")
const char* const kStageRange[] = {"rmesh/records",   "rmesh/project", "rmesh/tet_sort",
                                   "rmesh/emit",      "rmesh/pair_sort", "rmesh/ranges",
                                   "rmesh/composite", "rmesh/adam",    "rmesh/sh_adjoint"};

struct EventPair {
  int stage;
  cudaEvent_t a, b;
};

}  // namespace

struct RmeshCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int64_t N = 0, M = 0;
  int width = 0, height = 0, tile_size = 12;
  int tile_wide = 0;  // default tile configuration: tile_size, threads per tile doubled when set
  // per-resolution tile configurations (views of that size use them)
  struct ResConf {
    int W, H, ts, wide;
  };
  std::vector<ResConf> res_conf;
  int last_ts = 12, last_wide = 0;  // tile configuration of the last single-view forward
  float min_t = 0.0f;
  uint32_t step = 0;
  int sh_degree = -1;   // -1: base colours; 0..3: colours from SH coefficients
  int sh_nc = 0;        // (sh_degree + 1)^2
  float lr_sh = 0.0f;   // SH learning rate of rmesh_train_step
  int aux_dim = 0;      // custom per-tet aux channels
  std::string err;
  int num_sms = 148;

  // parameters + optimizer state
  DevBuf verts, idx, dens, cgrad, base, circ;
  DevBuf m_verts, v_verts, m_dens, v_dens, m_cgrad, v_cgrad, m_base, v_base;
  DevBuf rec, color4, grad_slot, csr_off, csr_ref;
  DevBuf sh, m_sh, v_sh;  // SH coefficients [M][3][nc] and their Adam moments
  DevBuf aux_data;        // [M][aux_dim] custom aux channels
  DevBuf dl_aux, d_aux;   // backward: [pixels][aux_dim] loss gradient, [M][aux_dim] data gradient

  // per-run
  DevBuf views_d, counters_d, hp_d, sort_state, sort_status, scan_status;
  // per (tet, view) item, at tet * n_views + view: tiles touched, projections,
  // tile-kernel record; compacted sort keys and values (item indices)
  DevBuf vis_key, vis_val, vis_cnt, vis_proj, vis_view, vis_key_alt, vis_val_alt, group_off;
  DevBuf vis_color, vis_dcolor;  // SH colours per entry and their gradients
  DevBuf pair_key, pair_val, pair_key_alt, pair_val_alt, ranges;
  DevBuf rgba, aux, dl, gt, out_a, out_b, out_c, out_d;
  DevBuf spans_fwd, spans_adj;  // per sorted pair: pixel spans of its tile rows (forward / adjoint rule)
  DevBuf tile_order, order_hist;  // longest-first tile order of the run; bucket counts and cursors
  DevBuf tickets;                 // persistent tile-queue heads, one per launch of a run
  DevBuf err_in, err_out;  // per-pixel error inputs, per-tet error statistics
  uint64_t cap_pairs = 0;
  uint64_t generation = 0;  // bumped whenever a buffer is reallocated

  // pinned host staging
  ViewParams* views_h = nullptr;
  Counters* counters_h = nullptr;
  AdamParams* hp_h = nullptr;

  // results of the last run
  uint32_t* sorted_pair_key = nullptr;
  uint32_t* sorted_pair_val = nullptr;
  bool have_forward = false;
  uint32_t last_tiles = 0;
  int last_views = 0;
  uint32_t last_err_bits = 0;
  uint64_t last_n_vis = 0, last_n_pairs = 0;
  int last_cnt = 1;  // Counters blocks written by the last training run

  // CUDA graphs of the batched train step, most recently used first; a step
  // whose signature (views, sizes, buffers, target pointer, ...) matches one
  // replays it, so callers alternating a few target buffers keep their graphs
  struct CachedGraph {
    std::vector<int64_t> sig;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;  // kernels per replay (counted at capture)
  };
  std::vector<CachedGraph> graphs;
  static constexpr size_t kMaxGraphs = 8;
  void drop_graphs() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }

  // profiling
  bool profiling = false;
  std::vector<EventPair> events;
  std::vector<cudaEvent_t> event_pool;
  float stage_ms[RMESH_N_STAGES] = {0};
  int stage_launches[RMESH_N_STAGES] = {0};
  int kernel_launches = 0;
};

namespace {

int fail(RmeshCtx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

// floats of the gradient buffer: 20 per tet, then (SH) 3 * nc per tet
size_t grad_floats(const RmeshCtx* c) { return (size_t)c->M * (kGradSlot + (c->sh_degree >= 0 ? 3 * c->sh_nc : 0)); }
float* sh_grad(const RmeshCtx* c) {
  return c->sh_degree >= 0 ? c->grad_slot.as<float>() + (size_t)c->M * kGradSlot : nullptr;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e__ = (call);                                                                     \
    if (e__ != cudaSuccess)                                                                       \
      return fail(c, e__ == cudaErrorMemoryAllocation ? RMESH_ERR_OOM : RMESH_ERR_CUDA,           \
                  std::string(#call) + ": " + cudaGetErrorString(e__));                           \
  } while (0)

#define CKL()                                                                                     \
  do {                                                                                            \
    cudaError_t e__ = cudaGetLastError();                                                         \
    if (e__ != cudaSuccess) return fail(c, RMESH_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e__)); \
    c->kernel_launches++;                                                                         \
  } while (0)

// One-time per-device settings.  cudaFuncSetAttribute applies to the current
// device only, so "already set" is recorded per device ordinal (under a mutex:
// contexts on different devices may be driven from different threads).
constexpr int kMaxDeviceOrdinals = 64;
struct PerDeviceOnce {
  std::mutex mu;
  bool done[kMaxDeviceOrdinals] = {};
  template <typename F>
  cudaError_t run(F f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDeviceOrdinals) return f();
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return cudaSuccess;
    e = f();
    if (e == cudaSuccess) done[dev] = true;
    return e;
  }
};

// Makes the context's device current for the duration of an API call and
// restores the caller's device afterwards (contexts on several devices can be
// driven from one thread).
struct DevGuard {
  int prev = -1;
  explicit DevGuard(const RmeshCtx* c) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
      return;
    }
    if (prev != c->device && cudaSetDevice(c->device) != cudaSuccess) cudaGetLastError();
  }
  ~DevGuard() {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
};

cudaEvent_t take_event(RmeshCtx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

struct StageScope {
  RmeshCtx* c;
  int stage;
  cudaEvent_t a = nullptr;
  bool ranged = false;
  StageScope(RmeshCtx* c_, int s, bool capturing) : c(c_), stage(s) {
    if (!capturing) {  // host-side range around the stage's launches
      nvtxRangePushA(kStageRange[s]);
      ranged = true;
    }
    if (c->profiling && !capturing) {
      a = take_event(c);
      cudaEventRecord(a, c->stream);
    }
  }
  ~StageScope() {
    if (a) {
      cudaEvent_t b = take_event(c);
      cudaEventRecord(b, c->stream);
      c->events.push_back({stage, a, b});
    }
    if (ranged) nvtxRangePop();
  }
};

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int bitlen(uint64_t x) {  // number of bits to represent x (x >= 1 -> >= 1)
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

int ensure_buf(RmeshCtx* c, DevBuf& b, size_t bytes) {
  bool grew = false;
  cudaError_t e = b.ensure(bytes, &grew);
  if (e != cudaSuccess) return fail(c, RMESH_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  if (grew) c->generation++;
  return RMESH_OK;
}

#define CKR(expr)              \
  do {                         \
    int r__ = (expr);          \
    if (r__ != RMESH_OK) return r__; \
  } while (0)

// ---------------------------------------------------------------- tile configurations
// A tile configuration: tile size 8, 12 or 16 and the threads per tile (one per
// pixel rounded up to whole warps, or twice that: WIDE).
struct TileConf {
  int ts = 12;
  int wide = 0;
  bool operator==(const TileConf& o) const { return ts == o.ts && wide == o.wide; }
};
constexpr int kMaxTileGroups = 8;

int conf_threads(TileConf t) { return (t.wide ? 2 : 1) * (((t.ts * t.ts + 31) / 32) * 32); }
int conf_minb(TileConf t) { return (t.wide ? 1 : 2) * (t.ts == 16 ? 1 : (t.ts == 12 ? 2 : 4)); }
bool conf_from(int ts, int threads, TileConf* out) {
  if (ts != 8 && ts != 12 && ts != 16) return false;
  TileConf t{ts, 0};
  if (threads == 0 || threads == conf_threads(t)) {
    *out = t;
    return true;
  }
  t.wide = 1;
  if (threads == conf_threads(t)) {
    *out = t;
    return true;
  }
  return false;
}

// the configuration a view of this size runs with
TileConf view_conf(const RmeshCtx* c, int W, int H) {
  for (const auto& r : c->res_conf)
    if (r.W == W && r.H == H) return TileConf{r.ts, r.wide};
  return TileConf{c->tile_size, c->tile_wide};
}

// Views of one tile configuration are numbered back to back (contiguous global
// tiles) and run as one persistent launch.
struct TileGroup {
  TileConf conf;
  uint32_t tile_lo = 0, n_tiles = 0;
};
struct ViewPlan {
  std::vector<int> order;        // order[i]: the caller's view placed at position i
  std::vector<TileConf> conf;    // per caller view
  std::vector<uint64_t> pix;     // first pixel of each caller view (caller order)
  std::vector<TileGroup> groups;
  uint64_t total_pix = 0;
  uint32_t total_tiles = 0, max_tiles = 0;
};

// ---------------------------------------------------------------- sorting
template <typename K>
int radix_sort(RmeshCtx* c, K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, const void* n_ptr, int n_is_u64,
               uint64_t cap, int bits, K** out_keys, uint32_t** out_vals, bool capturing) {
  const int passes = std::max(1, (bits + 7) / 8);
  SortState* st = c->sort_state.as<SortState>();
  Counters* cnt = c->counters_d.as<Counters>();
  CK(cudaMemsetAsync(st->hist, 0, sizeof(st->hist), c->stream));
  const int hist_blocks = (int)std::min<uint64_t>((cap + 255) / 256, (uint64_t)c->num_sms * 8);
  sort_hist_kernel<K><<<std::max(1, hist_blocks), 256, 0, c->stream>>>(keys, n_ptr, n_is_u64, cap, 0, passes, st);
  CKL();
  sort_scan_kernel<<<1, 256, 0, c->stream>>>(passes, st);
  CKL();
  constexpr int part = SortCfg<K>::PART;
  const size_t smem = sizeof(K) * part + sizeof(uint32_t) * part + sizeof(uint32_t) * (kSortWarps * 256 + 512);
  const unsigned grid = (unsigned)std::max<uint64_t>(1, (cap + part - 1) / part);
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int p = 0; p < passes; ++p) {
    onesweep_kernel<K><<<grid, kSortThreads, smem, c->stream>>>(kin, vin, kout, vout, n_ptr, n_is_u64, cap, 8 * p, p,
                                                                st, c->sort_status.as<unsigned long long>(),
                                                                &cnt->err);
    CKL();
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  (void)capturing;
  *out_keys = kin;
  *out_vals = vin;
  return RMESH_OK;
}

int setup_sort_attrs() {
  static PerDeviceOnce once;
  const cudaError_t e = once.run([]() -> cudaError_t {
    constexpr int p64 = SortCfg<uint64_t>::PART, p32 = SortCfg<uint32_t>::PART;
    const int s64 = (int)(sizeof(uint64_t) * p64 + sizeof(uint32_t) * p64 + sizeof(uint32_t) * (kSortWarps * 256 + 512));
    const int s32 = (int)(sizeof(uint32_t) * p32 + sizeof(uint32_t) * p32 + sizeof(uint32_t) * (kSortWarps * 256 + 512));
    cudaError_t r = cudaFuncSetAttribute(onesweep_kernel<unsigned long long>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(onesweep_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
  });
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return 0;
}

// ---------------------------------------------------------------- buffers
int ensure_run_buffers(RmeshCtx* c, int n_views, uint64_t total_pixels, uint32_t total_tiles) {
  const uint64_t items = (uint64_t)n_views * (uint64_t)c->M;
  CKR(ensure_buf(c, c->vis_key, items * 8));
  CKR(ensure_buf(c, c->vis_key_alt, items * 8));
  CKR(ensure_buf(c, c->vis_val, items * 4));
  CKR(ensure_buf(c, c->vis_val_alt, items * 4));
  CKR(ensure_buf(c, c->vis_cnt, items * 4));
  CKR(ensure_buf(c, c->group_off, ((items + 255) / 256 + 1) * 8));
  CKR(ensure_buf(c, c->vis_proj, items * 32));
  CKR(ensure_buf(c, c->vis_view, items * sizeof(TetView)));
  if (c->sh_degree >= 0) {
    CKR(ensure_buf(c, c->vis_color, items * 16));
    CKR(ensure_buf(c, c->vis_dcolor, items * 16));
  }
  if (c->cap_pairs == 0) c->cap_pairs = std::max<uint64_t>(8 * items, 1u << 16);
  CKR(ensure_buf(c, c->pair_key, c->cap_pairs * 4));
  CKR(ensure_buf(c, c->pair_val, c->cap_pairs * 4));
  CKR(ensure_buf(c, c->pair_key_alt, c->cap_pairs * 4));
  CKR(ensure_buf(c, c->pair_val_alt, c->cap_pairs * 4));
  CKR(ensure_buf(c, c->spans_fwd, c->cap_pairs * kSpanRec));
  CKR(ensure_buf(c, c->spans_adj, c->cap_pairs * kSpanRec));
  const uint64_t sort_items = std::max<uint64_t>(std::max<uint64_t>(items, c->cap_pairs), 4ull * c->M);
  CKR(ensure_buf(c, c->sort_status, ((sort_items + kSortPart - 1) / kSortPart + 1) * 256 * 8));
  CKR(ensure_buf(c, c->scan_status, ((items + 255) / 256 + 2) * 8));
  CKR(ensure_buf(c, c->ranges, (uint64_t)std::max<uint32_t>(total_tiles, 1) * 8));
  CKR(ensure_buf(c, c->tile_order, (uint64_t)std::max<uint32_t>(total_tiles, 1) * 4));
  CKR(ensure_buf(c, c->order_hist, 2 * kOrderBuckets * 4 * kMaxTileGroups));
  CKR(ensure_buf(c, c->tickets, kMaxTileGroups * 4));
  CKR(ensure_buf(c, c->rgba, std::max<uint64_t>(total_pixels, 1) * 16));
  return RMESH_OK;
}

// views_h[0..n) must be filled; uploads them
int upload_views(RmeshCtx* c, int n) {
  CK(cudaMemcpyAsync(c->views_d.p, c->views_h, sizeof(ViewParams) * n, cudaMemcpyHostToDevice, c->stream));
  return RMESH_OK;
}

int fill_view(RmeshCtx* c, const RmeshCamera& cam, ViewParams& v, uint32_t tile_base, uint32_t pix_base, TileConf tc) {
  if (cam.width <= 0 || cam.height <= 0 || cam.width > 65536 || cam.height > 65536)
    return fail(c, RMESH_ERR_INVALID_ARG, "camera width/height out of range");
  memset(&v, 0, sizeof(v));
  memcpy(v.vp, cam.vp, sizeof(v.vp));
  const float* ci = cam.c2w_intrinsics;
  for (int k = 0; k < 3; ++k) {
    v.c2w[k] = ci[k];
    v.c2w[3 + k] = ci[4 + k];
    v.c2w[6 + k] = ci[8 + k];
  }
  v.fx = ci[12];
  v.fy = ci[13];
  v.cx = ci[14];
  v.cy = ci[15];
  v.cam[0] = cam.cam_pos[0];
  v.cam[1] = cam.cam_pos[1];
  v.cam[2] = cam.cam_pos[2];
  v.min_t = c->min_t;
  v.W = cam.width;
  v.H = cam.height;
  v.Wf = (float)cam.width;
  v.Hf = (float)cam.height;
  v.n_pixels = (float)((uint32_t)cam.width * (uint32_t)cam.height);
  v.TS = tc.ts;
  v.tiles_x = (cam.width + tc.ts - 1) / tc.ts;
  v.tiles_y = (cam.height + tc.ts - 1) / tc.ts;
  v.tile_base = tile_base;
  v.pix_base = pix_base;
  return RMESH_OK;
}

// Fills views_h[0..n) in plan order (views of one configuration together) and
// the plan's groups.  plain: every view is its own run (tile ids from 0).
int make_plan(RmeshCtx* c, const RmeshCamera* cams, int n_views, bool plain, ViewPlan& pl) {
  pl = ViewPlan();
  pl.conf.resize(n_views);
  pl.pix.resize(n_views);
  std::vector<TileConf> distinct;
  for (int v = 0; v < n_views; ++v) {
    pl.conf[v] = view_conf(c, cams[v].width, cams[v].height);
    pl.pix[v] = pl.total_pix;
    pl.total_pix += (uint64_t)cams[v].width * cams[v].height;
    if (std::find(distinct.begin(), distinct.end(), pl.conf[v]) == distinct.end()) distinct.push_back(pl.conf[v]);
  }
  if ((int)distinct.size() > kMaxTileGroups) return fail(c, RMESH_ERR_INVALID_ARG, "too many tile configurations");
  if (pl.total_pix >= (1ull << 32)) return fail(c, RMESH_ERR_INVALID_ARG, "too many pixels in one run");
  for (const auto& tc : distinct) {
    TileGroup g;
    g.conf = tc;
    g.tile_lo = pl.total_tiles;
    for (int v = 0; v < n_views; ++v) {
      if (!(pl.conf[v] == tc)) continue;
      const int i = (int)pl.order.size();
      pl.order.push_back(v);
      CKR(fill_view(c, cams[v], c->views_h[i], plain ? 0u : pl.total_tiles, (uint32_t)pl.pix[v], tc));
      const uint32_t t = (uint32_t)(c->views_h[i].tiles_x * c->views_h[i].tiles_y);
      pl.total_tiles += t;
      pl.max_tiles = std::max(pl.max_tiles, t);
    }
    g.n_tiles = pl.total_tiles - g.tile_lo;
    pl.groups.push_back(g);
  }
  return RMESH_OK;
}

// ---------------------------------------------------------------- stages
int run_records(RmeshCtx* c, bool capturing) {
  StageScope sc(c, kStRecords, capturing);
  const int M = (int)c->M;
  build_records_kernel<<<(M + 255) / 256, 256, 0, c->stream>>>(M, c->verts.as<float>(), c->idx.as<uint4>(),
                                                               c->dens.as<float>(), c->cgrad.as<float>(),
                                                               c->base.as<float>(), c->rec.as<TetRec>(),
                                                               c->color4.as<float4>());
  CKL();
  return RMESH_OK;
}

// project -> tet sort -> emit -> pair sort -> ranges for n_views views at views_dev
int run_bin(RmeshCtx* c, const ViewParams* views_dev, int n_views, uint32_t total_tiles, Counters* cnt,
            bool capturing, const std::vector<TileGroup>& groups) {
  const uint64_t items = (uint64_t)n_views * (uint64_t)c->M;
  // chained scans over blocks of kCompactItems items (key compaction) and
  // sorted entries (pair offsets)
  const unsigned nscan = (unsigned)((items + kCompactItems - 1) / kCompactItems);
  unsigned long long* status = c->scan_status.as<unsigned long long>();
  uint32_t* ticket = reinterpret_cast<uint32_t*>(status + nscan + 1);
  {
    StageScope sc(c, kStProject, capturing);
    ProjectArgs pa;
    pa.M = (int)c->M;
    pa.n_views = n_views;
    pa.views = views_dev;
    pa.rec = c->rec.as<TetRec>();
    pa.vis_cnt = c->vis_cnt.as<uint32_t>();
    pa.vis_proj = c->vis_proj.as<float4>();
    pa.vis_view = c->vis_view.as<TetView>();
    pa.color4 = c->color4.as<float4>();
    pa.color_view_stride = 0;
    pa.sh = c->sh_degree >= 0 ? c->sh.as<float>() : nullptr;
    pa.sh_degree = c->sh_degree;
    pa.vis_color = c->vis_color.as<float4>();
    project_kernel<<<(unsigned)((items + 255) / 256), 256, 0, c->stream>>>(pa);
    CKL();
    CK(cudaMemsetAsync(status, 0, (size_t)(nscan + 2) * 8, c->stream));
    CompactArgs ca;
    ca.M = (int)c->M;
    ca.n_views = n_views;
    ca.views = views_dev;
    ca.circ = c->circ.as<float4>();
    ca.vis_cnt = c->vis_cnt.as<uint32_t>();
    ca.vis_key = c->vis_key.as<unsigned long long>();
    ca.vis_val = c->vis_val.as<uint32_t>();
    ca.status = status;
    ca.ticket = ticket;
    ca.counters = cnt;
    compact_keys_kernel<<<nscan, 256, 0, c->stream>>>(ca);
    CKL();
  }
  unsigned long long* tk = nullptr;
  uint32_t* tv = nullptr;
  {
    StageScope sc(c, kStTetSort, capturing);
    // depth bits only: pairs of different views never share a tile, so the
    // emission needs each view's entries in depth order (ties in item order,
    // i.e. by tet id), which a stable sort of all views' keys on depth alone
    // gives; the view and tile count ride in the key's high bits
    CKR(radix_sort<unsigned long long>(c, c->vis_key.as<unsigned long long>(), c->vis_val.as<uint32_t>(),
                                       c->vis_key_alt.as<unsigned long long>(), c->vis_val_alt.as<uint32_t>(),
                                       &cnt->n_vis, 0, items, 32, &tk, &tv, capturing));
  }
  {
    StageScope sc(c, kStEmit, capturing);
    CK(cudaMemsetAsync(status, 0, (size_t)(nscan + 2) * 8, c->stream));
    EmitScanArgs es;
    es.tet_key_sorted = tk;
    es.tet_val_sorted = tv;
    es.vis_cnt = c->vis_cnt.as<uint32_t>();
    es.n_vis_ptr = &cnt->n_vis;
    es.group_off = c->group_off.as<unsigned long long>();
    es.status = status;
    es.ticket = ticket;
    es.counters = cnt;
    emit_scan_kernel<<<nscan, 256, 0, c->stream>>>(es);
    CKL();
    EmitArgs ea;
    ea.views = views_dev;
    ea.tet_key_sorted = tk;
    ea.tet_val_sorted = tv;
    ea.vis_cnt = c->vis_cnt.as<uint32_t>();
    ea.vis_proj = c->vis_proj.as<float4>();
    ea.n_vis_ptr = &cnt->n_vis;
    ea.group_off = c->group_off.as<unsigned long long>();
    ea.pair_key = c->pair_key.as<uint32_t>();
    ea.pair_val = c->pair_val.as<uint32_t>();
    ea.cap = c->cap_pairs;
    ea.counters = cnt;
    emit_kernel<<<(unsigned)((items + 255) / 256), 256, 0, c->stream>>>(ea);
    CKL();
  }
  {
    StageScope sc(c, kStPairSort, capturing);
    const int bits = std::max(1, bitlen(total_tiles));
    CKR(radix_sort<uint32_t>(c, c->pair_key.as<uint32_t>(), c->pair_val.as<uint32_t>(), c->pair_key_alt.as<uint32_t>(),
                             c->pair_val_alt.as<uint32_t>(), &cnt->n_pairs, 1, c->cap_pairs, bits,
                             &c->sorted_pair_key, &c->sorted_pair_val, capturing));
  }
  {
    StageScope sc(c, kStRanges, capturing);
    CK(cudaMemsetAsync(c->ranges.p, 0, (size_t)total_tiles * 8, c->stream));
    const int blocks = (int)std::min<uint64_t>((c->cap_pairs + 255) / 256, (uint64_t)c->num_sms * 16);
    ranges_kernel<<<std::max(1, blocks), 256, 0, c->stream>>>(c->sorted_pair_key, &cnt->n_pairs, c->cap_pairs,
                                                               c->ranges.as<uint2>(), views_dev, n_views, cnt);
    CKL();
    PairSpanArgs sa;
    sa.views = views_dev;
    sa.n_views = n_views;
    sa.keys = c->sorted_pair_key;
    sa.vals = c->sorted_pair_val;
    sa.n_ptr = &cnt->n_pairs;
    sa.cap = c->cap_pairs;
    sa.vis_view = c->vis_view.as<TetView>();
    sa.spans_fwd = c->spans_fwd.as<uint8_t>();
    sa.spans_adj = c->spans_adj.as<uint8_t>();
    const int sblocks = (int)std::min<uint64_t>((c->cap_pairs + 255) / 256, (uint64_t)c->num_sms * 8);
    pair_spans_kernel<<<std::max(1, sblocks), 256, 0, c->stream>>>(sa);
    CKL();
    // longest-first order of each launch's tiles for the persistent tile
    // kernel (indices relative to the launch's first tile)
    CK(cudaMemsetAsync(c->order_hist.p, 0, 2 * kOrderBuckets * 4 * groups.size(), c->stream));
    CK(cudaMemsetAsync(c->tickets.p, 0, kMaxTileGroups * 4, c->stream));
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      const TileGroup& g = groups[gi];
      if (g.n_tiles == 0) continue;
      uint32_t* hist = c->order_hist.as<uint32_t>() + 2 * kOrderBuckets * gi;
      const int oblocks =
          (int)std::max<uint64_t>(1, std::min<uint64_t>((g.n_tiles + 255) / 256, (uint64_t)c->num_sms * 2));
      tile_order_hist_kernel<<<oblocks, 256, 0, c->stream>>>(c->ranges.as<uint2>() + g.tile_lo, g.n_tiles, hist);
      CKL();
      tile_order_stable_kernel<<<1, kOrderThreads, 0, c->stream>>>(c->ranges.as<uint2>() + g.tile_lo, g.n_tiles,
                                                                  hist, c->tile_order.as<uint32_t>() + g.tile_lo);
      CKL();
    }
  }
  return RMESH_OK;
}

template <int TS, int MODE, bool AUX, bool WIDE>
int launch_tile_t(RmeshCtx* c, TileArgs& ta, uint32_t n_tiles, bool persistent) {
  constexpr int NT = TileCfg<TS, AUX, WIDE>::NT;
  constexpr size_t smem = sizeof(TileSmem<TS, AUX, WIDE>);
  static PerDeviceOnce attrs;  // per instantiation and device
  CK(attrs.run([]() -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(tile_kernel<TS, MODE, AUX, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // the whole unified L1 as shared memory: resident CTAs are limited by it
    return cudaFuncSetAttribute(tile_kernel<TS, MODE, AUX, WIDE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
  }));
  unsigned grid = n_tiles;
  if (persistent) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tile_kernel<TS, MODE, AUX, WIDE>, NT, smem);
    grid = (unsigned)std::max(1, occ) * (unsigned)c->num_sms;
    grid = std::min<unsigned>(grid, std::max<uint32_t>(n_tiles, 1));
  }
  ta.persistent = persistent ? 1 : 0;
  if (grid == 0) return RMESH_OK;
  tile_kernel<TS, MODE, AUX, WIDE><<<grid, NT, smem, c->stream>>>(ta);
  CKL();
  return RMESH_OK;
}

// one launch over the tiles of a group (ta.tile_lo, ta.ticket set by the caller)
template <int MODE, bool AUX>
int launch_tile_m(RmeshCtx* c, TileArgs& ta, uint32_t n_tiles, bool persistent, TileConf tc) {
  const int key = tc.ts * 2 + (tc.wide ? 1 : 0);
  switch (key) {
    case 16: return launch_tile_t<8, MODE, AUX, false>(c, ta, n_tiles, persistent);
    case 17: return launch_tile_t<8, MODE, AUX, true>(c, ta, n_tiles, persistent);
    case 24: return launch_tile_t<12, MODE, AUX, false>(c, ta, n_tiles, persistent);
    case 25: return launch_tile_t<12, MODE, AUX, true>(c, ta, n_tiles, persistent);
    case 32: return launch_tile_t<16, MODE, AUX, false>(c, ta, n_tiles, persistent);
    case 33: return launch_tile_t<16, MODE, AUX, true>(c, ta, n_tiles, persistent);
    default: return fail(c, RMESH_ERR_INVALID_ARG, "tile size must be 8, 12 or 16");
  }
}

// one persistent launch per tile group of the run
template <int MODE, bool AUX>
int launch_groups(RmeshCtx* c, const TileArgs& base, const std::vector<TileGroup>& groups) {
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const TileGroup& g = groups[gi];
    if (g.n_tiles == 0) continue;
    TileArgs ta = base;
    ta.n_tiles = g.n_tiles;
    ta.tile_lo = g.tile_lo;
    ta.ticket = c->tickets.as<uint32_t>() + gi;
    ta.tile_order = c->tile_order.as<uint32_t>() + g.tile_lo;
    CKR((launch_tile_m<MODE, AUX>(c, ta, g.n_tiles, true, g.conf)));
  }
  return RMESH_OK;
}

TileArgs base_tile_args(RmeshCtx* c, const ViewParams* views_dev, int n_views, uint32_t n_tiles, Counters* cnt) {
  TileArgs ta;
  memset(&ta, 0, sizeof(ta));
  ta.views = views_dev;
  ta.n_views = n_views;
  ta.n_tiles = n_tiles;
  ta.ranges = c->ranges.as<uint2>();
  ta.pair_val = c->sorted_pair_val;
  ta.vis_view = c->vis_view.as<TetView>();
  ta.rec = c->rec.as<TetRec>();
  ta.color4 = c->color4.as<float4>();
  ta.color_view_stride = 0;
  ta.grad_slot = c->grad_slot.as<float>();
  if (c->sh_degree >= 0) {
    ta.vis_color = c->vis_color.as<float4>();
    ta.vis_dcolor = c->vis_dcolor.as<float4>();
  }
  ta.counters = cnt;
  ta.hp = c->hp_d.as<AdamParams>();
  ta.spans_fwd = c->spans_fwd.as<uint8_t>();
  ta.spans_adj = c->spans_adj.as<uint8_t>();
  ta.tile_order = c->tile_order.as<uint32_t>();
  ta.tile_lo = 0;
  ta.ticket = c->tickets.as<uint32_t>();
  return ta;
}

// SH colours: clears the per-entry colour gradients before an adjoint launch
int clear_dcolor(RmeshCtx* c, int n_views) {
  if (c->sh_degree < 0) return RMESH_OK;
  CK(cudaMemsetAsync(c->vis_dcolor.p, 0, (size_t)n_views * c->M * 16, c->stream));
  return RMESH_OK;
}

// SH colours: the adjoint of the colour evaluation, after an adjoint launch
int run_sh_backward(RmeshCtx* c, const ViewParams* views_dev, int n_views, bool capturing) {
  if (c->sh_degree < 0) return RMESH_OK;
  StageScope sc(c, kStShAdjoint, capturing);
  ShBackwardArgs sa;
  sa.M = (int)c->M;
  sa.n_views = n_views;
  sa.views = views_dev;
  sa.rec = c->rec.as<TetRec>();
  sa.sh = c->sh.as<float>();
  sa.vis_cnt = c->vis_cnt.as<uint32_t>();
  sa.vis_dcolor = c->vis_dcolor.as<float4>();
  sa.d_sh = sh_grad(c);
  sa.grad_slot = c->grad_slot.as<float>();
  const unsigned blocks = (unsigned)((c->M + 127) / 128);
  switch (c->sh_degree) {
    case 0: sh_backward_kernel<0><<<blocks, 128, 0, c->stream>>>(sa); break;
    case 1: sh_backward_kernel<1><<<blocks, 128, 0, c->stream>>>(sa); break;
    case 2: sh_backward_kernel<2><<<blocks, 128, 0, c->stream>>>(sa); break;
    default: sh_backward_kernel<3><<<blocks, 128, 0, c->stream>>>(sa); break;
  }
  CKL();
  return RMESH_OK;
}

int sync_counters(RmeshCtx* c, int n) {
  CK(cudaMemcpyAsync(c->counters_h, c->counters_d.p, sizeof(Counters) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  uint32_t bits = 0;
  uint64_t nv = 0, np = 0;
  for (int i = 0; i < n; ++i) {
    bits |= c->counters_h[i].err;
    nv += c->counters_h[i].n_vis;
    np = std::max<uint64_t>(np, c->counters_h[i].n_pairs);
  }
  c->last_err_bits = bits;
  c->last_n_vis = nv;
  c->last_n_pairs = np;
  return RMESH_OK;
}

// grows pair capacity after an overflow; returns true when a retry makes sense
bool grow_pairs(RmeshCtx* c) {
  const uint64_t need = c->last_n_pairs + c->last_n_pairs / 4 + 4096;
  const uint64_t limit = (1ull << 31) - 1;
  if (need <= c->cap_pairs || c->cap_pairs >= limit) return false;
  c->cap_pairs = std::min(need, limit);
  return true;
}

int status_from_bits(RmeshCtx* c) {
  if (c->last_err_bits & kErrSpinTimeout) return fail(c, RMESH_ERR_TIMEOUT, "device spin wait gave up");
  if (c->last_err_bits & kErrPairOverflow) return fail(c, RMESH_ERR_PAIR_OVERFLOW, "pair buffer overflow");
  return RMESH_OK;
}

int copy_in(RmeshCtx* c, DevBuf& dst, const void* src, size_t bytes) {
  if (!src || !bytes) return RMESH_OK;
  CK(cudaMemcpyAsync(dst.p, src, bytes, cudaMemcpyDefault, c->stream));
  return RMESH_OK;
}

// ---------------------------------------------------------------- train
int launch_adam(RmeshCtx* c, int n_cnt, bool capturing) {
  StageScope sc(c, kStAdam, capturing);
  AdamArgs aa;
  aa.N = (int)c->N;
  aa.M = (int)c->M;
  aa.verts = c->verts.as<float>();
  aa.dens = c->dens.as<float>();
  aa.cgrad = c->cgrad.as<float>();
  aa.base = c->base.as<float>();
  aa.m_verts = c->m_verts.as<float>();
  aa.v_verts = c->v_verts.as<float>();
  aa.m_dens = c->m_dens.as<float>();
  aa.v_dens = c->v_dens.as<float>();
  aa.m_cgrad = c->m_cgrad.as<float>();
  aa.v_cgrad = c->v_cgrad.as<float>();
  aa.m_base = c->m_base.as<float>();
  aa.v_base = c->v_base.as<float>();
  aa.grad_slot = c->grad_slot.as<float>();
  aa.sh = c->sh_degree >= 0 ? c->sh.as<float>() : nullptr;
  aa.m_sh = c->m_sh.as<float>();
  aa.v_sh = c->v_sh.as<float>();
  aa.d_sh = sh_grad(c);
  aa.n_sh = c->sh_degree >= 0 ? (long long)c->M * 3 * c->sh_nc : 0;
  aa.csr_off = c->csr_off.as<uint32_t>();
  aa.csr_ref = c->csr_ref.as<uint32_t>();
  aa.hp = c->hp_d.as<AdamParams>();
  aa.counters = c->counters_d.as<Counters>();
  aa.n_counters = n_cnt;
  const int blocks = (int)std::min<int64_t>((c->N + c->M + (aa.n_sh + 3) / 4 + 255) / 256, (int64_t)c->num_sms * 16);
  adam_kernel<<<std::max(1, blocks), 256, 0, c->stream>>>(aa);
  CKL();
  return RMESH_OK;
}

// Forward + loss + adjoint over n_views cameras, gradients summed into the
// per-tet slots; then (do_adam) one multi-group Adam launch.
int train_views(RmeshCtx* c, const RmeshCamera* cams, int n_views, const float* gt, const RmeshTrainOpts* o,
                float* loss_out, bool do_adam = true) {
  if (n_views <= 0 || n_views > kMaxViews) return fail(c, RMESH_ERR_INVALID_ARG, "n_views out of range");
  if (!cams || !gt || !o) return fail(c, RMESH_ERR_INVALID_ARG, "null argument");
  if (o->loss_type != 0 && o->loss_type != 1) return fail(c, RMESH_ERR_INVALID_ARG, "loss_type must be 0 or 1");
  const int mode = o->mode;
  const bool plain = mode == RMESH_MODE_PLAIN;
  // view table: batched numbering (tiles back to back, the views of each tile
  // configuration together; pixels in the caller's order)
  ViewPlan pl;
  CKR(make_plan(c, cams, n_views, plain, pl));
  const uint64_t total_pix = pl.total_pix;
  const uint32_t total_tiles = pl.total_tiles, max_tiles = pl.max_tiles;
  const int run_views = plain ? 1 : n_views;
  const bool direct_gt = is_device_ptr(gt);
  for (int attempt = 0; attempt < 4; ++attempt) {
    CKR(ensure_run_buffers(c, run_views, total_pix, plain ? max_tiles : total_tiles));
    if (!direct_gt) CKR(ensure_buf(c, c->gt, total_pix * 12));
    AdamParams& hp = *c->hp_h;
    hp.step = c->step + 1;
    hp.lr_verts = o->lr_verts;
    hp.lr_dens = o->lr_dens;
    hp.lr_grads = o->lr_grads;
    hp.lr_base = o->lr_base;
    hp.lr_sh = o->lr_sh;
    hp.beta1 = 0.9f;
    hp.beta2 = 0.999f;
    hp.eps = 1e-8f;
    hp.loss_type = o->loss_type;
    CK(cudaMemcpyAsync(c->hp_d.p, c->hp_h, sizeof(AdamParams), cudaMemcpyHostToDevice, c->stream));
    CKR(upload_views(c, n_views));
    const float* gt_dev = direct_gt ? gt : c->gt.as<float>();
    if (!direct_gt) CK(cudaMemcpyAsync(c->gt.p, gt, total_pix * 12, cudaMemcpyHostToDevice, c->stream));

    const int n_cnt = plain ? n_views : 1;
    auto enqueue = [&](bool capturing) -> int {
      Counters* cnt = c->counters_d.as<Counters>();
      CK(cudaMemsetAsync(cnt, 0, sizeof(Counters) * n_cnt, c->stream));
      CK(cudaMemsetAsync(c->grad_slot.p, 0, grad_floats(c) * 4, c->stream));
      CKR(run_records(c, capturing));
      ViewParams* vd = c->views_d.as<ViewParams>();
      if (plain) {
        for (int i = 0; i < n_views; ++i) {
          const uint32_t vt = (uint32_t)(c->views_h[i].tiles_x * c->views_h[i].tiles_y);
          const TileConf tc = pl.conf[pl.order[i]];
          const std::vector<TileGroup> one{TileGroup{tc, 0u, vt}};
          CKR(run_bin(c, vd + i, 1, vt, cnt + i, capturing, one));
          CKR(clear_dcolor(c, 1));
          {
            StageScope sc(c, kStComposite, capturing);
            TileArgs ta = base_tile_args(c, vd + i, 1, vt, cnt + i);
            ta.gt_rgb = gt_dev;
            CKR((launch_tile_m<kModeTrain, false>(c, ta, vt, false, tc)));
          }
          CKR(run_sh_backward(c, vd + i, 1, capturing));
        }
      } else {
        CKR(run_bin(c, vd, n_views, total_tiles, cnt, capturing, pl.groups));
        CKR(clear_dcolor(c, n_views));
        {
          StageScope sc(c, kStComposite, capturing);
          TileArgs ta = base_tile_args(c, vd, n_views, total_tiles, cnt);
          ta.gt_rgb = gt_dev;
          CKR((launch_groups<kModeTrain, false>(c, ta, pl.groups)));
        }
        CKR(run_sh_backward(c, vd, n_views, capturing));
      }
      if (do_adam) CKR(launch_adam(c, n_cnt, capturing));
      return RMESH_OK;
    };

    if (mode == RMESH_MODE_GRAPH) {
      std::vector<int64_t> sig = {n_views, 0, (int64_t)c->cap_pairs, (int64_t)c->generation,
                                  (int64_t)(uintptr_t)gt_dev, o->loss_type, do_adam ? 1 : 0};
      for (int v = 0; v < n_views; ++v) {
        sig.push_back(cams[v].width);
        sig.push_back(cams[v].height);
        sig.push_back(pl.conf[v].ts * 2 + pl.conf[v].wide);
      }
      // graphs captured before a reallocation point at freed buffers
      for (size_t i = c->graphs.size(); i-- > 0;)
        if (c->graphs[i].sig[3] != sig[3]) {
          cudaGraphExecDestroy(c->graphs[i].exec);
          c->graphs.erase(c->graphs.begin() + i);
        }
      size_t gi = 0;
      while (gi < c->graphs.size() && c->graphs[gi].sig != sig) ++gi;
      if (gi == c->graphs.size()) {
        RmeshCtx::CachedGraph cg;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int before = c->kernel_launches;
        int r = enqueue(true);
        cg.kernels = c->kernel_launches - before;
        c->kernel_launches = before;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (r != RMESH_OK) return r;
        if (e != cudaSuccess) return fail(c, RMESH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&cg.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(c, RMESH_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        cg.sig = sig;
        if (c->graphs.size() == RmeshCtx::kMaxGraphs) {
          cudaGraphExecDestroy(c->graphs.back().exec);
          c->graphs.pop_back();
        }
        c->graphs.insert(c->graphs.begin(), std::move(cg));
        gi = 0;
      } else if (gi > 0) {
        std::rotate(c->graphs.begin(), c->graphs.begin() + gi, c->graphs.begin() + gi + 1);
        gi = 0;
      }
      {
        StageScope sc(c, kStComposite, false);  // whole graph accounted as one span
        CK(cudaGraphLaunch(c->graphs[0].exec, c->stream));
        c->kernel_launches += c->graphs[0].kernels;
      }
    } else {
      CKR(enqueue(false));
    }
    CKR(sync_counters(c, n_cnt));
    if ((c->last_err_bits & kErrPairOverflow) && grow_pairs(c)) continue;
    CKR(status_from_bits(c));
    if (do_adam) c->step += 1;
    c->have_forward = false;
    c->last_cnt = n_cnt;
    if (loss_out) {
      for (int i = 0; i < n_views; ++i) {
        const int v = pl.order[i];
        const double l = plain ? c->counters_h[i].loss[0] : c->counters_h[0].loss[i];
        loss_out[v] = (float)(l / (double)((uint64_t)cams[v].width * cams[v].height));
      }
    }
    c->last_views = n_views;
    return RMESH_OK;
  }
  return fail(c, RMESH_ERR_PAIR_OVERFLOW, "pair buffers could not be grown enough");
}

int build_csr(RmeshCtx* c) {
  const uint64_t n_refs = 4ull * (uint64_t)c->M;
  CKR(ensure_buf(c, c->csr_off, (c->N + 1) * 4));
  CKR(ensure_buf(c, c->csr_ref, n_refs * 4));
  DevBuf k0, k1, v1, nbuf;
  CKR(ensure_buf(c, k0, n_refs * 4));
  CKR(ensure_buf(c, k1, n_refs * 4));
  CKR(ensure_buf(c, v1, n_refs * 4));
  CKR(ensure_buf(c, nbuf, 8));
  const uint32_t n32 = (uint32_t)n_refs;
  CK(cudaMemcpyAsync(nbuf.p, &n32, 4, cudaMemcpyHostToDevice, c->stream));
  csr_fill_kernel<<<(unsigned)((n_refs + 255) / 256), 256, 0, c->stream>>>((int)c->M, c->idx.as<uint32_t>(),
                                                                          k0.as<uint32_t>(), c->csr_ref.as<uint32_t>());
  CKL();
  CKR(ensure_buf(c, c->sort_status, ((n_refs + kSortPart - 1) / kSortPart + 1) * 256 * 8));
  CK(cudaMemsetAsync(c->counters_d.p, 0, sizeof(Counters), c->stream));
  uint32_t* ok_keys = nullptr;
  uint32_t* ok_vals = nullptr;
  CKR(radix_sort<uint32_t>(c, k0.as<uint32_t>(), c->csr_ref.as<uint32_t>(), k1.as<uint32_t>(), v1.as<uint32_t>(),
                           nbuf.p, 0, n_refs, std::max(1, bitlen((uint64_t)std::max<int64_t>(c->N - 1, 1))), &ok_keys,
                           &ok_vals, false));
  if (ok_vals != c->csr_ref.as<uint32_t>())
    CK(cudaMemcpyAsync(c->csr_ref.p, ok_vals, n_refs * 4, cudaMemcpyDeviceToDevice, c->stream));
  csr_offsets_kernel<<<(unsigned)((n_refs + 1 + 255) / 256), 256, 0, c->stream>>>((int)n_refs, (int)c->N, ok_keys,
                                                                                  c->csr_off.as<uint32_t>());
  CKL();
  CK(cudaStreamSynchronize(c->stream));
  Counters h;
  CK(cudaMemcpy(&h, c->counters_d.p, sizeof(Counters), cudaMemcpyDeviceToHost));
  if (h.err) return fail(c, RMESH_ERR_TIMEOUT, "vertex map sort failed");
  return RMESH_OK;
}

}  // namespace

// Exercises the two bounded waits of the path on conditions that never
// resolve: a chained-scan look-back whose predecessor never publishes
// (status[0] stays 0) and an mbarrier phase that never completes.  Each wait
// gives up after its limit and records kErrSpinTimeout in bits[0] / bits[1];
// the kernel then returns normally.
__global__ void timeout_probe_kernel(unsigned long long* status, uint32_t* bits) {
  __shared__ uint64_t bar;
  if (threadIdx.x < 32) chained_lookback(status, 1u, 1ull, &bits[0]);
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0u, 1u << 16)) atomicOr(&bits[1], kErrSpinTimeout);
}

// ===================================================================== C ABI
extern "C" {

int rmesh_abi_version(void) { return RMESH_ABI_VERSION; }

const char* rmesh_last_error(const RmeshCtx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int rmesh_create(const RmeshSceneDesc* d, RmeshCtx** out) {
  RmeshCtx* c = nullptr;
  if (!d || !out) return RMESH_ERR_INVALID_ARG;
  *out = nullptr;
  if (d->n_vertices <= 0 || d->n_tets <= 0 || !d->vertices || !d->indices || !d->base_colors || !d->densities ||
      !d->color_grads || !d->circumdata)
    return RMESH_ERR_INVALID_ARG;
  if (d->n_tets > (int64_t)(1u << 29) || d->n_vertices > (int64_t)(1u << 30)) return RMESH_ERR_INVALID_ARG;
  if (d->aux_dim < 0 || d->aux_dim > RMESH_MAX_AUX_DIM) return RMESH_ERR_INVALID_ARG;
  if (d->sh_coeffs && (d->sh_degree < 0 || d->sh_degree > 3)) return RMESH_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RMESH_ERR_NO_DEVICE;
  }
  c = new RmeshCtx();
  c->N = d->n_vertices;
  c->M = d->n_tets;
  c->width = d->width;
  c->height = d->height;
  c->tile_size = d->tile_size > 0 ? d->tile_size : 12;
  c->aux_dim = d->aux_dim;
  if (d->sh_coeffs) {
    c->sh_degree = d->sh_degree;
    c->sh_nc = (d->sh_degree + 1) * (d->sh_degree + 1);
  }
  if (c->tile_size != 8 && c->tile_size != 12 && c->tile_size != 16) {
    delete c;
    return RMESH_ERR_INVALID_ARG;
  }
  if (d->device >= 0) {
    if (cudaSetDevice(d->device) != cudaSuccess) {
      delete c;
      return RMESH_ERR_NO_DEVICE;
    }
  }
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  if (setup_sort_attrs() != 0) {
    delete c;
    return RMESH_ERR_NO_DEVICE;
  }
  int r = RMESH_OK;
  auto init = [&]() -> int {
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    CK(cudaMallocHost(&c->views_h, sizeof(ViewParams) * kMaxViews));
    CK(cudaMallocHost(&c->counters_h, sizeof(Counters) * kMaxViews));
    CK(cudaMallocHost(&c->hp_h, sizeof(AdamParams)));
    const size_t N = (size_t)c->N, M = (size_t)c->M;
    CKR(ensure_buf(c, c->verts, 3 * N * 4));
    CKR(ensure_buf(c, c->idx, 4 * M * 4));
    CKR(ensure_buf(c, c->dens, M * 4));
    CKR(ensure_buf(c, c->cgrad, 3 * M * 4));
    CKR(ensure_buf(c, c->base, 3 * M * 4));
    CKR(ensure_buf(c, c->circ, 4 * M * 4));
    DevBuf* zeros[] = {&c->m_verts, &c->v_verts, &c->m_dens, &c->v_dens, &c->m_cgrad, &c->v_cgrad, &c->m_base, &c->v_base};
    size_t zsz[] = {3 * N, 3 * N, M, M, 3 * M, 3 * M, 3 * M, 3 * M};
    for (int i = 0; i < 8; ++i) {
      CKR(ensure_buf(c, *zeros[i], zsz[i] * 4));
      CK(cudaMemsetAsync(zeros[i]->p, 0, zsz[i] * 4, c->stream));
    }
    CKR(ensure_buf(c, c->rec, M * sizeof(TetRec)));
    CKR(ensure_buf(c, c->color4, M * 16));
    CKR(ensure_buf(c, c->grad_slot, grad_floats(c) * 4));
    if (c->aux_dim > 0) {
      CKR(ensure_buf(c, c->aux_data, M * (size_t)c->aux_dim * 4));
      CK(cudaMemsetAsync(c->aux_data.p, 0, M * (size_t)c->aux_dim * 4, c->stream));
    }
    if (c->sh_degree >= 0) {
      const size_t n_sh = M * 3 * (size_t)c->sh_nc;
      CKR(ensure_buf(c, c->sh, n_sh * 4));
      CKR(ensure_buf(c, c->m_sh, n_sh * 4));
      CKR(ensure_buf(c, c->v_sh, n_sh * 4));
      CK(cudaMemsetAsync(c->m_sh.p, 0, n_sh * 4, c->stream));
      CK(cudaMemsetAsync(c->v_sh.p, 0, n_sh * 4, c->stream));
      CKR(copy_in(c, c->sh, d->sh_coeffs, n_sh * 4));
    }
    CKR(ensure_buf(c, c->views_d, sizeof(ViewParams) * kMaxViews));
    CKR(ensure_buf(c, c->counters_d, sizeof(Counters) * kMaxViews));
    CKR(ensure_buf(c, c->hp_d, sizeof(AdamParams)));
    CKR(ensure_buf(c, c->sort_state, sizeof(SortState)));
    CK(cudaMemsetAsync(c->sort_state.p, 0, sizeof(SortState), c->stream));
    CKR(copy_in(c, c->verts, d->vertices, 3 * N * 4));
    CKR(copy_in(c, c->idx, d->indices, 4 * M * 4));
    {
      // every index must name a vertex before any kernel gathers through it
      uint32_t* bad = c->counters_d.as<uint32_t>();  // scratch word; the counters are cleared per run
      CK(cudaMemsetAsync(bad, 0, 4, c->stream));
      const int blocks = (int)std::min<uint64_t>((4 * M + 255) / 256, (uint64_t)c->num_sms * 8);
      index_range_kernel<<<std::max(1, blocks), 256, 0, c->stream>>>(c->idx.as<uint32_t>(), 4 * (uint64_t)M,
                                                                     (uint32_t)N, bad);
      CKL();
      uint32_t bad_h = 0;
      CK(cudaMemcpyAsync(&bad_h, bad, 4, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (bad_h) return fail(c, RMESH_ERR_INVALID_ARG, "a tet index is not below the vertex count");
    }
    CKR(copy_in(c, c->dens, d->densities, M * 4));
    CKR(copy_in(c, c->cgrad, d->color_grads, 3 * M * 4));
    CKR(copy_in(c, c->base, d->base_colors, 3 * M * 4));
    CKR(copy_in(c, c->circ, d->circumdata, 4 * M * 4));
    CKR(build_csr(c));
    return RMESH_OK;
  };
  r = init();
  if (r != RMESH_OK) {
    rmesh_destroy(c);
    return r;
  }
  *out = c;
  return RMESH_OK;
}

int rmesh_destroy(RmeshCtx* c) {
  if (!c) return RMESH_OK;
  DevGuard dg__(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->drop_graphs();
  for (auto& e : c->events) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  if (c->views_h) cudaFreeHost(c->views_h);
  if (c->counters_h) cudaFreeHost(c->counters_h);
  if (c->hp_h) cudaFreeHost(c->hp_h);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return RMESH_OK;
}

int rmesh_set_stream(RmeshCtx* c, void* s) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  CK(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->own_stream = false;
  c->stream = (cudaStream_t)s;
  c->drop_graphs();
  return RMESH_OK;
}

int rmesh_set_min_t(RmeshCtx* c, float t) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  c->min_t = t;
  return RMESH_OK;
}

int rmesh_set_tile_size(RmeshCtx* c, int32_t ts) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (ts != 8 && ts != 12 && ts != 16) return fail(c, RMESH_ERR_INVALID_ARG, "tile size must be 8, 12 or 16");
  c->tile_size = ts;
  c->tile_wide = 0;
  c->have_forward = false;
  return RMESH_OK;
}

int rmesh_set_tile_config(RmeshCtx* c, int32_t ts, int32_t threads) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  TileConf tc;
  if (!conf_from(ts, threads, &tc)) return fail(c, RMESH_ERR_INVALID_ARG, "unsupported tile size / threads per tile");
  c->tile_size = tc.ts;
  c->tile_wide = tc.wide;
  c->have_forward = false;
  return RMESH_OK;
}

int rmesh_set_resolution_tile_config(RmeshCtx* c, int32_t width, int32_t height, int32_t ts, int32_t threads) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  auto& rc = c->res_conf;
  rc.erase(std::remove_if(rc.begin(), rc.end(), [&](const RmeshCtx::ResConf& r) { return r.W == width && r.H == height; }),
           rc.end());
  c->have_forward = false;
  if (ts == 0) return RMESH_OK;  // override removed
  TileConf tc;
  if (!conf_from(ts, threads, &tc)) return fail(c, RMESH_ERR_INVALID_ARG, "unsupported tile size / threads per tile");
  rc.push_back(RmeshCtx::ResConf{width, height, tc.ts, tc.wide});
  return RMESH_OK;
}

int rmesh_get_tile_config(RmeshCtx* c, int32_t width, int32_t height, int32_t* ts, int32_t* threads) {
  if (!c || !ts || !threads) return RMESH_ERR_INVALID_ARG;
  const TileConf tc = (width > 0 && height > 0) ? view_conf(c, width, height) : TileConf{c->tile_size, c->tile_wide};
  *ts = tc.ts;
  *threads = conf_threads(tc);
  return RMESH_OK;
}

int rmesh_update_params(RmeshCtx* c, const float* v, const float* b, const float* d, const float* g) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  CKR(copy_in(c, c->verts, v, 3 * (size_t)c->N * 4));
  CKR(copy_in(c, c->base, b, 3 * (size_t)c->M * 4));
  CKR(copy_in(c, c->dens, d, (size_t)c->M * 4));
  CKR(copy_in(c, c->cgrad, g, 3 * (size_t)c->M * 4));
  return RMESH_OK;
}

int rmesh_get_params(RmeshCtx* c, float* v, float* b, float* d, float* g) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (v) CK(cudaMemcpyAsync(v, c->verts.p, 3 * (size_t)c->N * 4, cudaMemcpyDefault, c->stream));
  if (b) CK(cudaMemcpyAsync(b, c->base.p, 3 * (size_t)c->M * 4, cudaMemcpyDefault, c->stream));
  if (d) CK(cudaMemcpyAsync(d, c->dens.p, (size_t)c->M * 4, cudaMemcpyDefault, c->stream));
  if (g) CK(cudaMemcpyAsync(g, c->cgrad.p, 3 * (size_t)c->M * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_set_aux_data(RmeshCtx* c, const float* aux_data) {
  if (!c || !aux_data) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (c->aux_dim == 0) return fail(c, RMESH_ERR_INVALID_ARG, "aux_dim is 0; create the context with aux_dim > 0");
  CKR(copy_in(c, c->aux_data, aux_data, (size_t)c->M * c->aux_dim * 4));
  return RMESH_OK;
}

int rmesh_get_aux_data(RmeshCtx* c, float* aux_data) {
  if (!c || !aux_data) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (c->aux_dim == 0) return fail(c, RMESH_ERR_INVALID_ARG, "aux_dim is 0; no aux data");
  CK(cudaMemcpyAsync(aux_data, c->aux_data.p, (size_t)c->M * c->aux_dim * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_set_lr_sh(RmeshCtx* c, float lr) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  c->lr_sh = lr;
  return RMESH_OK;
}

int rmesh_update_sh(RmeshCtx* c, const float* sh) {
  if (!c || !sh) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (c->sh_degree < 0) return fail(c, RMESH_ERR_STATE, "the context has no SH coefficients");
  CKR(copy_in(c, c->sh, sh, (size_t)c->M * 3 * c->sh_nc * 4));
  return RMESH_OK;
}

int rmesh_get_sh(RmeshCtx* c, float* sh) {
  if (!c || !sh) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (c->sh_degree < 0) return fail(c, RMESH_ERR_STATE, "the context has no SH coefficients");
  CK(cudaMemcpyAsync(sh, c->sh.p, (size_t)c->M * 3 * c->sh_nc * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_get_sh_grad(RmeshCtx* c, float* d_sh) {
  if (!c || !d_sh) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (c->sh_degree < 0) return fail(c, RMESH_ERR_STATE, "the context has no SH coefficients");
  CK(cudaMemcpyAsync(d_sh, sh_grad(c), (size_t)c->M * 3 * c->sh_nc * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_get_info(RmeshCtx* c, RmeshInfo* info) {
  if (!c || !info) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  memset(info, 0, sizeof(*info));
  info->n_vertices = c->N;
  info->n_tets = c->M;
  info->width = c->width;
  info->height = c->height;
  info->tile_size = c->tile_size;
  info->n_views_last = c->last_views;
  info->step = c->step;
  info->last_error_bits = c->last_err_bits;
  info->n_visible_last = c->last_n_vis;
  info->n_pairs_last = c->last_n_pairs;
  info->pair_capacity = c->cap_pairs;
  DevBuf* all[] = {&c->verts, &c->idx, &c->dens, &c->cgrad, &c->base, &c->circ, &c->m_verts, &c->v_verts,
                   &c->m_dens, &c->v_dens, &c->m_cgrad, &c->v_cgrad, &c->m_base, &c->v_base, &c->rec,
                   &c->color4, &c->grad_slot, &c->csr_off, &c->csr_ref, &c->views_d, &c->counters_d, &c->hp_d,
                   &c->sort_state, &c->sort_status, &c->scan_status, &c->vis_key, &c->vis_val, &c->group_off,
                   &c->vis_cnt, &c->vis_proj, &c->vis_view, &c->vis_key_alt, &c->vis_val_alt, &c->pair_key,
                   &c->pair_val, &c->pair_key_alt, &c->pair_val_alt, &c->ranges, &c->rgba, &c->aux, &c->dl,
                   &c->gt, &c->out_a, &c->out_b, &c->out_c, &c->out_d, &c->sh, &c->m_sh, &c->v_sh,
                   &c->vis_color, &c->vis_dcolor, &c->err_in, &c->err_out, &c->aux_data, &c->dl_aux, &c->d_aux,
                   &c->spans_fwd, &c->spans_adj, &c->tile_order, &c->order_hist, &c->tickets};
  for (DevBuf* b : all) info->device_bytes += b->bytes;
  return RMESH_OK;
}

// the Adam moment buffers in checkpoint order, with their lengths in floats
static std::vector<std::pair<DevBuf*, uint64_t>> adam_state_parts(RmeshCtx* c) {
  const uint64_t N = (uint64_t)c->N, M = (uint64_t)c->M;
  std::vector<std::pair<DevBuf*, uint64_t>> parts = {
      {&c->m_verts, 3 * N}, {&c->v_verts, 3 * N}, {&c->m_dens, M},     {&c->v_dens, M},
      {&c->m_cgrad, 3 * M}, {&c->v_cgrad, 3 * M}, {&c->m_base, 3 * M}, {&c->v_base, 3 * M}};
  if (c->sh_degree >= 0) {
    const uint64_t n_sh = 3 * (uint64_t)c->sh_nc * M;
    parts.push_back({&c->m_sh, n_sh});
    parts.push_back({&c->v_sh, n_sh});
  }
  return parts;
}

int rmesh_adam_state_size(RmeshCtx* c, uint64_t* n_floats) {
  if (!c || !n_floats) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  uint64_t n = 0;
  for (auto& p : adam_state_parts(c)) n += p.second;
  *n_floats = n;
  return RMESH_OK;
}

int rmesh_get_adam_state(RmeshCtx* c, float* state, uint32_t* step) {
  if (!c || !state) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  uint64_t off = 0;
  for (auto& p : adam_state_parts(c)) {
    CK(cudaMemcpyAsync(state + off, p.first->p, p.second * 4, cudaMemcpyDefault, c->stream));
    off += p.second;
  }
  CK(cudaStreamSynchronize(c->stream));
  if (step) *step = c->step;
  return RMESH_OK;
}

int rmesh_set_adam_state(RmeshCtx* c, const float* state, uint32_t step) {
  if (!c || !state) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  uint64_t off = 0;
  for (auto& p : adam_state_parts(c)) {
    CK(cudaMemcpyAsync(p.first->p, state + off, p.second * 4, cudaMemcpyDefault, c->stream));
    off += p.second;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->step = step;
  return RMESH_OK;
}

int rmesh_forward_views(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, float* rgba_out, float* aux_out) {
  if (!c || !cams || !rgba_out) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (n_views <= 0 || n_views > kMaxViews) return fail(c, RMESH_ERR_INVALID_ARG, "n_views out of range");
  ViewPlan pl;
  CKR(make_plan(c, cams, n_views, false, pl));
  const uint64_t total_pix = pl.total_pix;
  const uint32_t total_tiles = pl.total_tiles;
  const uint64_t aux_floats = total_pix * (8 + (uint64_t)c->aux_dim);
  for (int attempt = 0; attempt < 4; ++attempt) {
    CKR(ensure_run_buffers(c, n_views, total_pix, total_tiles));
    if (aux_out) CKR(ensure_buf(c, c->aux, aux_floats * 4));
    CKR(upload_views(c, n_views));
    Counters* cnt = c->counters_d.as<Counters>();
    CK(cudaMemsetAsync(cnt, 0, sizeof(Counters), c->stream));
    CKR(run_records(c, false));
    ViewParams* vd = c->views_d.as<ViewParams>();
    CKR(run_bin(c, vd, n_views, total_tiles, cnt, false, pl.groups));
    {
      StageScope sc(c, kStComposite, false);
      TileArgs ta = base_tile_args(c, vd, n_views, total_tiles, cnt);
      ta.rgba = c->rgba.as<float>();
      if (aux_out) {
        ta.aux = c->aux.as<float>();
        ta.aux_data = c->aux_data.as<float>();
        ta.aux_dim = c->aux_dim;
        CKR((launch_groups<kModeForward, true>(c, ta, pl.groups)));
      } else {
        CKR((launch_groups<kModeForward, false>(c, ta, pl.groups)));
      }
    }
    CKR(sync_counters(c, 1));
    if ((c->last_err_bits & kErrPairOverflow) && grow_pairs(c)) continue;
    CKR(status_from_bits(c));
    CK(cudaMemcpyAsync(rgba_out, c->rgba.p, total_pix * 16, cudaMemcpyDefault, c->stream));
    if (aux_out) CK(cudaMemcpyAsync(aux_out, c->aux.p, aux_floats * 4, cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->have_forward = false;
    c->last_views = n_views;
    return RMESH_OK;
  }
  return fail(c, RMESH_ERR_PAIR_OVERFLOW, "pair buffers could not be grown enough");
}

int rmesh_forward_tiled(RmeshCtx* c, const RmeshCamera* cam, float* rgba_out, float* aux_out) {
  if (!c || !cam || !rgba_out) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  const uint64_t npix = (uint64_t)cam->width * cam->height;
  const TileConf tc = view_conf(c, cam->width, cam->height);
  for (int attempt = 0; attempt < 4; ++attempt) {
    CKR(fill_view(c, *cam, c->views_h[0], 0, 0, tc));
    const uint32_t tiles = (uint32_t)(c->views_h[0].tiles_x * c->views_h[0].tiles_y);
    const std::vector<TileGroup> one{TileGroup{tc, 0u, tiles}};
    CKR(ensure_run_buffers(c, 1, npix, tiles));
    if (aux_out) CKR(ensure_buf(c, c->aux, npix * (8 + (uint64_t)c->aux_dim) * 4));
    CKR(upload_views(c, 1));
    Counters* cnt = c->counters_d.as<Counters>();
    CK(cudaMemsetAsync(cnt, 0, sizeof(Counters), c->stream));
    CKR(run_records(c, false));
    ViewParams* vd = c->views_d.as<ViewParams>();
    CKR(run_bin(c, vd, 1, tiles, cnt, false, one));
    {
      StageScope sc(c, kStComposite, false);
      TileArgs ta = base_tile_args(c, vd, 1, tiles, cnt);
      ta.rgba = c->rgba.as<float>();
      if (aux_out) {
        ta.aux = c->aux.as<float>();
        ta.aux_data = c->aux_data.as<float>();
        ta.aux_dim = c->aux_dim;
        CKR((launch_groups<kModeForward, true>(c, ta, one)));
      } else {
        CKR((launch_groups<kModeForward, false>(c, ta, one)));
      }
    }
    CKR(sync_counters(c, 1));
    if ((c->last_err_bits & kErrPairOverflow) && grow_pairs(c)) continue;
    CKR(status_from_bits(c));
    CK(cudaMemcpyAsync(rgba_out, c->rgba.p, npix * 16, cudaMemcpyDefault, c->stream));
    if (aux_out) CK(cudaMemcpyAsync(aux_out, c->aux.p, npix * (8 + (uint64_t)c->aux_dim) * 4, cudaMemcpyDefault, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->have_forward = true;
    c->last_tiles = tiles;
    c->last_views = 1;
    c->last_ts = tc.ts;
    c->last_wide = tc.wide;
    return RMESH_OK;
  }
  return fail(c, RMESH_ERR_PAIR_OVERFLOW, "pair buffers could not be grown enough");
}

// rmesh_backward and rmesh_backward_aux: dl_aux / d_aux only with aux channels
static int backward_impl(RmeshCtx* c, const float* dl, const float* dl_aux, float* d_verts, float* d_dens,
                         float* d_base, float* d_cgrad, float* d_aux) {
  if (!c->have_forward) return fail(c, RMESH_ERR_STATE, "backward() must follow forward_tiled()");
  const ViewParams& v = c->views_h[0];
  const uint64_t npix = (uint64_t)v.W * v.H;
  const bool with_aux = c->aux_dim > 0 && (dl_aux || d_aux);
  CKR(ensure_buf(c, c->dl, npix * 16));
  CK(cudaMemcpyAsync(c->dl.p, dl, npix * 16, cudaMemcpyDefault, c->stream));
  CK(cudaMemsetAsync(c->grad_slot.p, 0, grad_floats(c) * 4, c->stream));
  if (with_aux) {
    CKR(ensure_buf(c, c->dl_aux, npix * (uint64_t)c->aux_dim * 4));
    CKR(ensure_buf(c, c->d_aux, (uint64_t)c->M * c->aux_dim * 4));
    if (dl_aux)
      CK(cudaMemcpyAsync(c->dl_aux.p, dl_aux, npix * (uint64_t)c->aux_dim * 4, cudaMemcpyDefault, c->stream));
    else
      CK(cudaMemsetAsync(c->dl_aux.p, 0, npix * (uint64_t)c->aux_dim * 4, c->stream));
    CK(cudaMemsetAsync(c->d_aux.p, 0, (uint64_t)c->M * c->aux_dim * 4, c->stream));
  }
  Counters* cnt = c->counters_d.as<Counters>();
  CK(cudaMemsetAsync(c->tickets.p, 0, kMaxTileGroups * 4, c->stream));
  const std::vector<TileGroup> one{TileGroup{TileConf{c->last_ts, c->last_wide}, 0u, c->last_tiles}};
  ViewParams* vd = c->views_d.as<ViewParams>();
  CKR(clear_dcolor(c, 1));
  {
    StageScope sc(c, kStComposite, false);
    TileArgs ta = base_tile_args(c, vd, 1, c->last_tiles, cnt);
    ta.rgba = c->rgba.as<float>();
    ta.dl_rgba = c->dl.as<float>();
    if (with_aux) {
      ta.aux_data = c->aux_data.as<float>();
      ta.aux_dim = c->aux_dim;
      ta.dl_aux = c->dl_aux.as<float>();
      ta.d_aux = c->d_aux.as<float>();
      CKR((launch_groups<kModeBackward, true>(c, ta, one)));
    } else {
      CKR((launch_groups<kModeBackward, false>(c, ta, one)));
    }
  }
  if (d_aux && with_aux)
    CK(cudaMemcpyAsync(d_aux, c->d_aux.p, (uint64_t)c->M * c->aux_dim * 4, cudaMemcpyDefault, c->stream));
  CKR(run_sh_backward(c, vd, 1, false));
  const size_t N = (size_t)c->N, M = (size_t)c->M;
  CKR(ensure_buf(c, c->out_a, 3 * N * 4));
  CKR(ensure_buf(c, c->out_b, M * 4));
  CKR(ensure_buf(c, c->out_c, 3 * M * 4));
  CKR(ensure_buf(c, c->out_d, 3 * M * 4));
  const int blocks = (int)std::min<int64_t>((c->N + c->M + 255) / 256, (int64_t)c->num_sms * 16);
  unpack_grads_kernel<<<std::max(1, blocks), 256, 0, c->stream>>>(
      (int)c->N, (int)c->M, c->grad_slot.as<float>(), c->csr_off.as<uint32_t>(), c->csr_ref.as<uint32_t>(),
      c->out_a.as<float>(), c->out_b.as<float>(), c->out_c.as<float>(), c->out_d.as<float>());
  CKL();
  if (d_verts) CK(cudaMemcpyAsync(d_verts, c->out_a.p, 3 * N * 4, cudaMemcpyDefault, c->stream));
  if (d_dens) CK(cudaMemcpyAsync(d_dens, c->out_b.p, M * 4, cudaMemcpyDefault, c->stream));
  if (d_base) CK(cudaMemcpyAsync(d_base, c->out_c.p, 3 * M * 4, cudaMemcpyDefault, c->stream));
  if (d_cgrad) CK(cudaMemcpyAsync(d_cgrad, c->out_d.p, 3 * M * 4, cudaMemcpyDefault, c->stream));
  CKR(sync_counters(c, 1));
  return status_from_bits(c);
}

int rmesh_backward(RmeshCtx* c, const float* dl, float* d_verts, float* d_dens, float* d_base, float* d_cgrad) {
  if (!c || !dl) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  return backward_impl(c, dl, nullptr, d_verts, d_dens, d_base, d_cgrad, nullptr);
}

int rmesh_backward_aux(RmeshCtx* c, const float* dl, const float* dl_aux, float* d_verts, float* d_dens,
                       float* d_base, float* d_cgrad, float* d_aux) {
  if (!c || !dl) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  return backward_impl(c, dl, dl_aux, d_verts, d_dens, d_base, d_cgrad, d_aux);
}

int rmesh_forward_error(RmeshCtx* c, const float* pixel_err, const float* ssim_err, float* tet_err,
                        int32_t* tet_count) {
  if (!c || !pixel_err || !ssim_err || !tet_err || !tet_count) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!c->have_forward) return fail(c, RMESH_ERR_STATE, "forward_error() must follow forward_tiled()");
  const ViewParams& v = c->views_h[0];
  const uint64_t npix = (uint64_t)v.W * v.H;
  const size_t M = (size_t)c->M;
  CKR(ensure_buf(c, c->err_in, npix * 8));
  CKR(ensure_buf(c, c->err_out, M * 18 * 4));
  float* pe = c->err_in.as<float>();
  CK(cudaMemcpyAsync(pe, pixel_err, npix * 4, cudaMemcpyDefault, c->stream));
  CK(cudaMemcpyAsync(pe + npix, ssim_err, npix * 4, cudaMemcpyDefault, c->stream));
  CK(cudaMemsetAsync(c->err_out.p, 0, M * 18 * 4, c->stream));
  Counters* cnt = c->counters_d.as<Counters>();
  CK(cudaMemsetAsync(c->tickets.p, 0, kMaxTileGroups * 4, c->stream));
  const std::vector<TileGroup> one{TileGroup{TileConf{c->last_ts, c->last_wide}, 0u, c->last_tiles}};
  ViewParams* vd = c->views_d.as<ViewParams>();
  {
    StageScope sc(c, kStComposite, false);
    TileArgs ta = base_tile_args(c, vd, 1, c->last_tiles, cnt);
    ta.pixel_err = pe;
    ta.ssim_err = pe + npix;
    ta.tet_err = c->err_out.as<float>();
    ta.tet_count = reinterpret_cast<int*>(c->err_out.as<float>() + M * 16);
    CKR((launch_groups<kModeError, false>(c, ta, one)));
  }
  CK(cudaMemcpyAsync(tet_err, c->err_out.p, M * 16 * 4, cudaMemcpyDefault, c->stream));
  CK(cudaMemcpyAsync(tet_count, c->err_out.as<float>() + M * 16, M * 8, cudaMemcpyDefault, c->stream));
  CKR(sync_counters(c, 1));
  return status_from_bits(c);
}

int rmesh_train_step(RmeshCtx* c, const RmeshCamera* cam, const float* gt, float lr_verts, float lr_dens,
                     float lr_grads, int32_t loss_type, float* loss_out) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  RmeshTrainOpts o;
  memset(&o, 0, sizeof(o));
  o.lr_verts = lr_verts;
  o.lr_dens = lr_dens;
  o.lr_grads = lr_grads;
  o.lr_base = 0.0f;
  o.lr_sh = c->lr_sh;
  o.loss_type = loss_type;
  o.mode = RMESH_MODE_BATCHED;
  return train_views(c, cam, 1, gt, &o, loss_out);
}

int rmesh_train_step_views(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, const float* gt,
                           const RmeshTrainOpts* opts, float* loss_out) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!opts || opts->mode < 0 || opts->mode > 2) return fail(c, RMESH_ERR_INVALID_ARG, "bad mode");
  return train_views(c, cams, n_views, gt, opts, loss_out);
}

int rmesh_accumulate_views(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, const float* gt,
                           const RmeshTrainOpts* opts, float* loss_out) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!opts || opts->mode < 0 || opts->mode > 2) return fail(c, RMESH_ERR_INVALID_ARG, "bad mode");
  return train_views(c, cams, n_views, gt, opts, loss_out, false);
}

}  // extern "C"

namespace {

// ms per batched forward + loss + adjoint run (no Adam: parameters unchanged)
// of these views at the context's current tile configurations: one warm-up
// run (sizes the buffers), then two timed runs
int time_views(RmeshCtx* c, const RmeshCamera* cams, int n, const float* gt, const RmeshTrainOpts& o,
               cudaEvent_t e0, cudaEvent_t e1, float* ms) {
  c->have_forward = false;
  CKR(train_views(c, cams, n, gt, &o, nullptr, false));
  CK(cudaEventRecord(e0, c->stream));
  for (int r = 0; r < 2; ++r) CKR(train_views(c, cams, n, gt, &o, nullptr, false));
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(ms, e0, e1));
  *ms *= 0.5f;
  return RMESH_OK;
}

int autotune_impl(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, const float* gt, const RmeshTrainOpts* opts,
                  bool wide_too, bool per_resolution, std::vector<RmeshTuneEntry>& out) {
  RmeshTrainOpts o = *opts;
  o.mode = RMESH_MODE_BATCHED;
  std::vector<TileConf> grid;
  for (int ts : {8, 12, 16})
    for (int w = 0; w < (wide_too ? 2 : 1); ++w) grid.push_back(TileConf{ts, w});
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evg{e0, e1};
  c->res_conf.clear();
  // every configuration on all views
  TileConf best{c->tile_size, c->tile_wide};
  float best_ms = 0.f;
  for (size_t i = 0; i < grid.size(); ++i) {
    c->tile_size = grid[i].ts;
    c->tile_wide = grid[i].wide;
    float ms = 0.f;
    CKR(time_views(c, cams, n_views, gt, o, e0, e1, &ms));
    out.push_back(RmeshTuneEntry{0, 0, grid[i].ts, conf_threads(grid[i]), ms});
    if (i == 0 || ms < best_ms) {
      best_ms = ms;
      best = grid[i];
    }
  }
  c->tile_size = best.ts;
  c->tile_wide = best.wide;
  // every configuration on the views of each resolution; a resolution whose
  // best configuration differs from the overall best gets an override, kept
  // only if the mixed step beats the best single configuration
  std::vector<std::pair<int, int>> res;
  for (int v = 0; v < n_views; ++v) {
    const std::pair<int, int> r{cams[v].width, cams[v].height};
    if (std::find(res.begin(), res.end(), r) == res.end()) res.push_back(r);
  }
  if (!per_resolution || res.size() < 2) return RMESH_OK;
  std::vector<RmeshCtx::ResConf> chosen;
  for (const auto& r : res) {
    std::vector<RmeshCamera> sub;
    for (int v = 0; v < n_views; ++v)
      if (cams[v].width == r.first && cams[v].height == r.second) sub.push_back(cams[v]);
    TileConf rb = best;
    float rb_ms = 0.f;
    for (size_t i = 0; i < grid.size(); ++i) {
      c->tile_size = grid[i].ts;
      c->tile_wide = grid[i].wide;
      float ms = 0.f;
      CKR(time_views(c, sub.data(), (int)sub.size(), gt, o, e0, e1, &ms));
      out.push_back(RmeshTuneEntry{r.first, r.second, grid[i].ts, conf_threads(grid[i]), ms});
      if (i == 0 || ms < rb_ms) {
        rb_ms = ms;
        rb = grid[i];
      }
    }
    if (!(rb == best)) chosen.push_back(RmeshCtx::ResConf{r.first, r.second, rb.ts, rb.wide});
  }
  c->tile_size = best.ts;
  c->tile_wide = best.wide;
  if (chosen.empty()) return RMESH_OK;
  c->res_conf = chosen;
  float mixed_ms = 0.f;
  CKR(time_views(c, cams, n_views, gt, o, e0, e1, &mixed_ms));
  out.push_back(RmeshTuneEntry{-1, -1, 0, 0, mixed_ms});
  if (mixed_ms >= best_ms) c->res_conf.clear();
  return RMESH_OK;
}

}  // namespace

extern "C" {

int rmesh_autotune(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, const float* gt,
                   const RmeshTrainOpts* opts, int32_t per_resolution, RmeshTuneEntry* entries, int32_t max_entries,
                   int32_t* n_entries) {
  if (!c || !cams || !gt || !opts || !n_entries || (max_entries > 0 && !entries)) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  std::vector<RmeshTuneEntry> out;
  const int rc = autotune_impl(c, cams, n_views, gt, opts, true, per_resolution != 0, out);
  c->have_forward = false;
  *n_entries = (int32_t)out.size();
  for (int i = 0; i < (int)out.size() && i < max_entries; ++i) entries[i] = out[i];
  return rc;
}

int rmesh_autotune_tile_size(RmeshCtx* c, const RmeshCamera* cams, int32_t n_views, const float* gt,
                             const RmeshTrainOpts* opts, int32_t* tile_size_out, float* ms_out) {
  if (!c || !cams || !gt || !opts || !tile_size_out) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  std::vector<RmeshTuneEntry> out;
  const int rc = autotune_impl(c, cams, n_views, gt, opts, false, false, out);
  c->have_forward = false;
  for (size_t i = 0; i < out.size() && i < 3; ++i)
    if (ms_out) ms_out[i] = out[i].ms;
  *tile_size_out = c->tile_size;
  return rc;
}

int rmesh_grad_slots(RmeshCtx* c, float** ptr, uint64_t* n_floats) {
  if (!c || !ptr || !n_floats) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  *ptr = c->grad_slot.as<float>();
  *n_floats = grad_floats(c);
  return RMESH_OK;
}

int rmesh_apply_adam(RmeshCtx* c, const RmeshTrainOpts* o) {
  if (!c || !o) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  AdamParams& hp = *c->hp_h;
  hp.step = c->step + 1;
  hp.lr_verts = o->lr_verts;
  hp.lr_dens = o->lr_dens;
  hp.lr_grads = o->lr_grads;
  hp.lr_base = o->lr_base;
  hp.lr_sh = o->lr_sh;
  hp.beta1 = 0.9f;
  hp.beta2 = 0.999f;
  hp.eps = 1e-8f;
  hp.loss_type = o->loss_type;
  CK(cudaMemcpyAsync(c->hp_d.p, c->hp_h, sizeof(AdamParams), cudaMemcpyHostToDevice, c->stream));
  CKR(launch_adam(c, c->last_cnt, false));
  CK(cudaStreamSynchronize(c->stream));
  c->step += 1;
  return RMESH_OK;
}

int rmesh_debug_tiles_touched(RmeshCtx* c, uint32_t* out) {
  if (!c || !out) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!c->have_forward) return fail(c, RMESH_ERR_STATE, "no forward yet");
  // the single-view forward's items are the tet ids
  CK(cudaMemcpyAsync(out, c->vis_cnt.p, (size_t)c->M * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_debug_pairs(RmeshCtx* c, uint32_t* tiles, uint32_t* tets, uint64_t cap, uint64_t* n) {
  if (!c || !n) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!c->have_forward) return fail(c, RMESH_ERR_STATE, "no forward yet");
  *n = c->last_n_pairs;
  const uint64_t k = std::min<uint64_t>(cap, c->last_n_pairs);
  if (k && tiles) CK(cudaMemcpyAsync(tiles, c->sorted_pair_key, k * 4, cudaMemcpyDefault, c->stream));
  if (k && tets) {
    // the pair payload is the item index tet * n_views + view: map it to tet
    // ids in the pair buffer the sort left free
    uint32_t* scratch = c->sorted_pair_val == c->pair_val.as<uint32_t>() ? c->pair_val_alt.as<uint32_t>()
                                                                          : c->pair_val.as<uint32_t>();
    const int blocks = (int)std::min<uint64_t>((k + 255) / 256, (uint64_t)c->num_sms * 8);
    pair_tets_kernel<<<blocks, 256, 0, c->stream>>>(c->sorted_pair_key, c->sorted_pair_val,
                                                     (uint32_t)std::max(c->last_views, 1), k, scratch);
    CKL();
    CK(cudaMemcpyAsync(tets, scratch, k * 4, cudaMemcpyDefault, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_debug_ranges(RmeshCtx* c, uint32_t* ranges, uint64_t n_tiles) {
  if (!c || !ranges) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  if (!c->have_forward) return fail(c, RMESH_ERR_STATE, "no forward yet");
  const uint64_t k = std::min<uint64_t>(n_tiles, c->last_tiles);
  CK(cudaMemcpyAsync(ranges, c->ranges.p, k * 8, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return RMESH_OK;
}

int rmesh_debug_timeouts(uint32_t* bits_out) {
  if (!bits_out) return RMESH_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RMESH_ERR_NO_DEVICE;
  }
  void* buf = nullptr;
  if (cudaMalloc(&buf, 64) != cudaSuccess) return RMESH_ERR_OOM;
  int rc = RMESH_OK;
  if (cudaMemset(buf, 0, 64) != cudaSuccess) rc = RMESH_ERR_CUDA;
  if (rc == RMESH_OK) {
    timeout_probe_kernel<<<1, 64>>>(reinterpret_cast<unsigned long long*>(buf),
                                    reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + 32));
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(bits_out, static_cast<char*>(buf) + 32, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = RMESH_ERR_CUDA;
  }
  cudaFree(buf);
  return rc;
}

int rmesh_set_profiling(RmeshCtx* c, int32_t on) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  c->profiling = on != 0;
  return RMESH_OK;
}

int rmesh_stage_times(RmeshCtx* c, float* ms_out, int32_t* launches_out) {
  if (!c) return RMESH_ERR_INVALID_ARG;
  DevGuard dg__(c);
  CK(cudaStreamSynchronize(c->stream));
  for (auto& e : c->events) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
      c->stage_ms[e.stage] += ms;
      c->stage_launches[e.stage] += 1;
    }
    c->event_pool.push_back(e.a);
    c->event_pool.push_back(e.b);
  }
  c->events.clear();
  if (ms_out)
    for (int i = 0; i < RMESH_N_STAGES; ++i) ms_out[i] = c->stage_ms[i];
  if (launches_out) {
    for (int i = 0; i < RMESH_N_STAGES; ++i) launches_out[i] = c->stage_launches[i];
    launches_out[RMESH_N_STAGES] = c->kernel_launches;
  }
  for (int i = 0; i < RMESH_N_STAGES; ++i) {
    c->stage_ms[i] = 0.f;
    c->stage_launches[i] = 0;
  }
  c->kernel_launches = 0;
  return RMESH_OK;
}

}  // extern "C"

// ============================================================================
// Allocation-free tile count (rmesh_count_tiles_static)
//
// For callers that must not allocate device memory: a per-frame visibility
// query in an interactive viewer, where cudaMalloc / cudaFree would
// synchronise the device mid-frame, or a caller with a fixed device-memory
// budget that owns no renderer context (a context allocates every buffer of
// the path).  The entry point runs a variant of project_kernel (the same cull,
// the same conservative tile count and the same chained-scan compaction of the
// tile-touching tets) whose only scratch, the scan's block ticket and status
// words, lives in the fixed file-scope array below.  It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Every call on a device shares that device's array.  The ticket and the first
// ceil(n_tets / 256) status words must start at zero; each call clears them
// with a memset on its own stream before its launch.  Two calls in flight at
// the same time on one device (other streams, other threads) race on the array
// and return wrong results: order them on one stream or with events.
// ============================================================================
namespace rm {

constexpr uint32_t kStaticMaxTets = RMESH_STATIC_MAX_TETS;
constexpr uint32_t kStaticScanBlocks = kStaticMaxTets / 256u;
constexpr size_t kStaticTicketBytes = 256;  // the block ticket, on its own 256-byte line
constexpr size_t kStaticScratchBytes = kStaticTicketBytes + 8 * (size_t)kStaticScanBlocks;  // 524,544 bytes
constexpr uint32_t kErrBadIndex = 1u << 2;  // a vertex index >= n_vertices (the tet is skipped)
static_assert(kStaticMaxTets % 256u == 0, "scan positions");

static __device__ __align__(256) unsigned char g_count_scratch[kStaticScratchBytes];

// Single-view variant of project_kernel: gathers the four vertices and the
// density of each tet straight from the mesh arrays (no per-tet records), and
// writes tiles_touched by tet id plus the ids of the tile-touching tets in
// ascending order.  counts[0] receives their number, counts[1] error bits.
__global__ void __launch_bounds__(256) count_tiles_static_kernel(const float* __restrict__ verts, uint64_t n_verts,
                                                                 const uint32_t* __restrict__ idx,
                                                                 const float* __restrict__ dens, uint32_t M,
                                                                 ViewParams V, uint32_t* __restrict__ tiles_touched,
                                                                 uint32_t* __restrict__ visible, uint32_t* counts,
                                                                 unsigned char* scratch) {
  uint32_t* ticket = reinterpret_cast<uint32_t*>(scratch);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(scratch + kStaticTicketBytes);
  __shared__ uint32_t s_blk;
  __shared__ uint32_t s_warp[8];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_blk = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint32_t blk = s_blk;
  const uint32_t tet = blk * 256u + threadIdx.x;

  uint32_t count = 0;
  bool flag = false, bad = false;
  if (tet < M) {
    uint32_t q[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      q[k] = idx[4 * (size_t)tet + k];
      bad = bad || (uint64_t)q[k] >= n_verts;
    }
    bool visible = !bad;
    if (!bad) {
      float vx[4], vy[4], vz[4], p[4][4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        vx[k] = verts[3 * (size_t)q[k]];
        vy[k] = verts[3 * (size_t)q[k] + 1];
        vz[k] = verts[3 * (size_t)q[k] + 2];
        float c[4];
        clip_exact(V.vp, vx[k], vy[k], vz[k], c);
        const float inv_w = fdv(1.0f, fa(c[3], 1e-6f));
        p[k][0] = fm(c[0], inv_w);
        p[k][1] = fm(c[1], inv_w);
        p[k][2] = fm(c[2], inv_w);
        p[k][3] = c[3];
      }
      const bool any_behind = (p[0][3] <= 0.0f) || (p[1][3] <= 0.0f) || (p[2][3] <= 0.0f) || (p[3][3] <= 0.0f);
      if (!any_behind) {  // NDC box and extent culls (project_compute.wgsl:124-144)
        const float min_x = fminf(fminf(p[0][0], p[1][0]), fminf(p[2][0], p[3][0]));
        const float max_x = fmaxf(fmaxf(p[0][0], p[1][0]), fmaxf(p[2][0], p[3][0]));
        const float min_y = fminf(fminf(p[0][1], p[1][1]), fminf(p[2][1], p[3][1]));
        const float max_y = fmaxf(fmaxf(p[0][1], p[1][1]), fmaxf(p[2][1], p[3][1]));
        const float min_z = fminf(fminf(p[0][2], p[1][2]), fminf(p[2][2], p[3][2]));
        if (max_x < -1.0f || min_x > 1.0f || max_y < -1.0f || min_y > 1.0f || min_z > 1.0f) visible = false;
        if (fm(fm(fs(max_x, min_x), V.Wf), fm(fs(max_y, min_y), V.Hf)) < 1.0f) visible = false;
      }
      if (visible) {  // optical-depth cull (project_compute.wgsl:146-162)
        const int ei[6] = {1, 2, 3, 2, 3, 3};
        const int ej[6] = {0, 0, 0, 1, 1, 2};
        float e2[6];
#pragma unroll
        for (int e = 0; e < 6; ++e) {
          const float dx = fs(vx[ei[e]], vx[ej[e]]), dy = fs(vy[ei[e]], vy[ej[e]]), dz = fs(vz[ei[e]], vz[ej[e]]);
          e2[e] = dot3x(dx, dy, dz, dx, dy, dz);
        }
        const float m = fmaxf(fmaxf(e2[0], fmaxf(e2[1], e2[2])), fmaxf(e2[3], fmaxf(e2[4], e2[5])));
        if (fm(dens[tet], __fsqrt_rn(m)) < 0.01f) visible = false;
      }
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
    }
    if (!visible) count = 0u;
    tiles_touched[tet] = count;
    flag = count > 0u;
  }
  if (bad) atomicOr(&counts[1], kErrBadIndex);
  // block scan of the flags, then the chained scan across blocks
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned ballot = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) s_warp[warp] = __popc(ballot);
  __syncthreads();
  uint32_t warp_off = 0, block_total = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const uint32_t c = s_warp[w];
    if (w < warp) warp_off += c;
    block_total += c;
  }
  if (warp == 0) {
    const unsigned long long pre = chained_lookback(status, blk, block_total, &counts[1]);
    if (lane == 0) s_prefix = pre;
  }
  __syncthreads();
  const unsigned long long base = s_prefix;
  if (flag) visible[base + warp_off + __popc(ballot & ((1u << lane) - 1u))] = tet;
  if (threadIdx.x == 0 && (uint64_t)(blk + 1u) * 256u >= M) counts[0] = (uint32_t)(base + block_total);
}

namespace {

// Device address of g_count_scratch per device ordinal, looked up by every
// call made with that device current.
constexpr int kStaticMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_ptr[kStaticMaxDevices] = {};

typedef int (*MemRangeFn)(unsigned long long* base, size_t* size, unsigned long long ptr);

// [p, p + bytes) must lie in one device (or managed) allocation of the current
// device; the kernel would otherwise read or write outside the caller's arrays.
bool device_range_ok(const void* p, size_t bytes, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeDevice) {
    if (at.device != dev) return false;
  } else if (at.type != cudaMemoryTypeManaged) {
    return false;
  }
  // looked up once; a function-local static initialiser is thread-safe
  static const MemRangeFn range_fn = []() -> MemRangeFn {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<MemRangeFn>(fn);
    cudaGetLastError();
    return nullptr;
  }();
  if (range_fn) {
    unsigned long long base = 0;
    size_t size = 0;
    if (range_fn(&base, &size, (unsigned long long)(uintptr_t)p) != 0) return false;
    if ((uintptr_t)p + bytes > base + size) return false;
  }
  return true;
}

}  // namespace
}  // namespace rm

extern "C" int rmesh_count_tiles_static(const float* vertices, uint64_t n_vertices, const uint32_t* indices,
                                        const float* densities, uint64_t n_tets, const RmeshCamera* cam,
                                        int32_t tile_size, uint32_t* tiles_touched, uint32_t* visible_tets,
                                        uint32_t* counts, void* stream) {
  using namespace rm;
  if (n_tets > kStaticMaxTets) return RMESH_ERR_TOO_LARGE;
  if (!cam || !counts) return RMESH_ERR_INVALID_ARG;
  if (n_tets > 0 && (!vertices || !indices || !densities || !tiles_touched || !visible_tets || n_vertices == 0))
    return RMESH_ERR_INVALID_ARG;
  if (n_vertices > (1ull << 32)) return RMESH_ERR_INVALID_ARG;
  const int ts = tile_size == 0 ? 12 : tile_size;
  if (ts < 1 || ts > 256) return RMESH_ERR_INVALID_ARG;
  if (cam->width <= 0 || cam->height <= 0 || cam->width > 65536 || cam->height > 65536) return RMESH_ERR_INVALID_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return RMESH_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kStaticMaxDevices) return RMESH_ERR_INVALID_ARG;
  unsigned char* scratch = nullptr;
  {
    // The scratch array's device address on this device.  The first call on a
    // device may load the module there, so make it before any stream capture.
    // The address is looked up again on every call (cheap once the module is
    // loaded), so a device reset between calls cannot leave a stale pointer;
    // the cached copy only records that the first lookup happened.
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_count_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return RMESH_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    scratch = g_scratch_ptr[dev];
  }

  const uint64_t M = n_tets;
  if (!device_range_ok(counts, 8, dev)) return RMESH_ERR_INVALID_ARG;
  if (M > 0 && (!device_range_ok(vertices, 12 * n_vertices, dev) || !device_range_ok(indices, 16 * M, dev) ||
                !device_range_ok(densities, 4 * M, dev) || !device_range_ok(tiles_touched, 4 * M, dev) ||
                !device_range_ok(visible_tets, 4 * M, dev)))
    return RMESH_ERR_INVALID_ARG;

  ViewParams V;
  memset(&V, 0, sizeof(V));
  memcpy(V.vp, cam->vp, sizeof(V.vp));
  V.cam[0] = cam->cam_pos[0];
  V.cam[1] = cam->cam_pos[1];
  V.cam[2] = cam->cam_pos[2];
  V.W = cam->width;
  V.H = cam->height;
  V.Wf = (float)cam->width;
  V.Hf = (float)cam->height;
  V.TS = ts;
  V.tiles_x = (cam->width + ts - 1) / ts;
  V.tiles_y = (cam->height + ts - 1) / ts;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counts, 0, 8, st) != cudaSuccess) {
    cudaGetLastError();
    return RMESH_ERR_CUDA;
  }
  if (M == 0) return RMESH_OK;
  const uint32_t nblk = (uint32_t)((M + 255) / 256);
  if (cudaMemsetAsync(scratch, 0, kStaticTicketBytes + 8 * (size_t)nblk, st) != cudaSuccess) {
    cudaGetLastError();
    return RMESH_ERR_CUDA;
  }
  count_tiles_static_kernel<<<nblk, 256, 0, st>>>(vertices, n_vertices, indices, densities, (uint32_t)M, V,
                                                   tiles_touched, visible_tets, counts, scratch);
  if (cudaGetLastError() != cudaSuccess) return RMESH_ERR_CUDA;
  return RMESH_OK;
}

// ============================================================================
// .rmesh scene decode (rmesh_decode_scene): the host slices the file into its
// sections and uploads them; the kernels in rmesh_file.cuh decode them.
// ============================================================================
extern "C" int rmesh_decode_scene(const RmeshPackedScene* in, float* densities, float* color_grads, float* sh_coeffs,
                                  float* circumdata, void* stream) {
  using namespace rm;
  if (!in || !densities || !color_grads || !sh_coeffs || !circumdata) return RMESH_ERR_INVALID_ARG;
  if (in->n_tets == 0 || in->n_vertices == 0 || in->sh_degree > 3 || in->n_tets > (1ull << 31))
    return RMESH_ERR_INVALID_ARG;
  if (!in->vertices || !in->indices || !in->log_densities || !in->sh_mean || !in->sh_basis || !in->sh_weights)
    return RMESH_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return RMESH_ERR_NO_DEVICE;
  }
  const uint64_t M = in->n_tets, N = in->n_vertices;
  const uint32_t nc = (in->sh_degree + 1) * (in->sh_degree + 1), D = 3 * nc;
  const uint32_t K = std::min<uint32_t>(in->k_components, D);
  if (!device_range_ok(in->vertices, 12 * N, dev) || !device_range_ok(in->indices, 16 * M, dev) ||
      !device_range_ok(in->log_densities, M, dev) || !device_range_ok(in->sh_mean, 2ull * D, dev) ||
      (K > 0 && !device_range_ok(in->sh_basis, 2ull * K * D, dev)) ||
      (K > 0 && !device_range_ok(in->sh_weights, 2ull * K * M, dev)) ||
      (in->color_grads && !device_range_ok(in->color_grads, 6 * M, dev)) || !device_range_ok(densities, 4 * M, dev) ||
      !device_range_ok(color_grads, 12 * M, dev) || !device_range_ok(sh_coeffs, 4ull * D * M, dev) ||
      !device_range_ok(circumdata, 16 * M, dev))
    return RMESH_ERR_INVALID_ARG;
  SceneDecodeArgs a;
  a.M = M;
  a.D = D;
  a.K = K;
  a.verts = in->vertices;
  a.idx = in->indices;
  a.log_dens = in->log_densities;
  a.mean = in->sh_mean;
  a.basis = in->sh_basis;
  a.weights = in->sh_weights;
  a.grads16 = in->color_grads;
  a.dens = densities;
  a.grads = color_grads;
  a.sh = sh_coeffs;
  a.circ = reinterpret_cast<float4*>(circumdata);
  for (int i = 0; i < 256; ++i) a.table.v[i] = std::exp(((float)i - 100.0f) / 20.0f);  // the loader's f32 expf
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned b1 = (unsigned)std::min<uint64_t>((M + 255) / 256, 65535ull * 8);
  decode_tets_kernel<<<b1, 256, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return RMESH_ERR_CUDA;
  const unsigned b2 = (unsigned)std::min<uint64_t>((M * D + 255) / 256, 65535ull * 8);
  pca_decode_kernel<<<b2, 256, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return RMESH_ERR_CUDA;
  return RMESH_OK;
}
