// Tile binning: emit (tile, tet) pairs in depth order, then per-tile ranges.
//
// Order of work (B200 design): tets are first sorted by ~depth at tet
// granularity (onesweep over the 32 depth bits of all views' entries at once:
// pairs of different views never share a tile, so each view's entries in
// depth order suffice; the view and tile count ride in the key's high bits),
// then each tet emits its tiles at offsets given by a scan of
// tiles_touched in that order (emit_scan_kernel), and a short
// stable sort on the global tile id (ceil(log2 tiles) bits) finishes the job.
// Per tile this yields exactly the reference's order -- ascending 64-bit key
// (tile << 32 | ~depth) with ties broken by tet id -- while the pair-level sort
// touches 2-3 digits instead of the reference's 6-7
// (crates/rmesh-sort/src/drs.rs:23-26).
//
// Emission restates crates/rmesh-tile/src/wgsl/tile_gen_scan_compute.wgsl:61-203:
// division-projected vertices, at most tiles_touched pairs per tet (the count
// project_compute.wgsl made with multiply-by-reciprocal projection), and a
// sentinel (tile 0xFFFFFFFF, value 0) for every slot the tet leaves unfilled
// (tile_fill_compute.wgsl:9-19).  Sentinels sort after every real tile.
#pragma once
#include "common.cuh"
#include "project.cuh"

namespace rm {

// Pair offsets of the sorted entries: a chained scan of their tile counts in
// sorted order over blocks of kCompactItems entries (kCompactPerThread
// consecutive entries per thread).  It writes the exclusive offset of every
// 256-entry group (the emission kernel's blocks; group g of a scan block is
// warp g's entries) and the total pair count.
struct EmitScanArgs {
  const unsigned long long* tet_key_sorted;  // count << 40 | view << 32 | ~depth, sorted
  const uint32_t* tet_val_sorted;            // item index
  const uint32_t* vis_cnt;                   // counts of items whose key count saturated
  const uint32_t* n_vis_ptr;
  unsigned long long* group_off;             // [ceil(n / 256)] exclusive pair offset of each group
  unsigned long long* status;
  uint32_t* ticket;
  Counters* counters;
};

__device__ __forceinline__ uint32_t key_count(unsigned long long key, uint32_t val, const uint32_t* vis_cnt) {
  const uint32_t c = (uint32_t)(key >> 40);
  return c < kKeyCountMax ? c : vis_cnt[val];
}

__global__ void __launch_bounds__(256) emit_scan_kernel(EmitScanArgs a) {
  __shared__ uint32_t s_blk;
  __shared__ unsigned long long s_warp[8];
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_blk = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const uint32_t blk = s_blk;
  const uint32_t n = *a.n_vis_ptr;
  if ((unsigned long long)blk * kCompactItems >= n) return;  // later blocks never wait on this one
  const unsigned long long k0 = (unsigned long long)blk * kCompactItems + (unsigned long long)threadIdx.x * kCompactPerThread;
  unsigned long long mine = 0;
#pragma unroll
  for (int q = 0; q < kCompactPerThread; ++q)
    if (k0 + q < n) mine += key_count(a.tet_key_sorted[k0 + q], a.tet_val_sorted[k0 + q], a.vis_cnt);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long x = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  unsigned long long woff = 0, btot = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    if (w < warp) woff += s_warp[w];
    btot += s_warp[w];
  }
  if (warp == 0) {
    const unsigned long long pre = chained_lookback(a.status, blk, btot, &a.counters->err);
    if (lane == 0) s_prefix = pre;
  }
  __syncthreads();
  const unsigned long long group = (unsigned long long)blk * (kCompactItems / 256) + (unsigned long long)warp;
  if (lane == 0 && group * 256ull < n) a.group_off[group] = s_prefix + woff;
  if (threadIdx.x == 0 && (unsigned long long)(blk + 1) * kCompactItems >= n) a.counters->n_pairs = s_prefix + btot;
}

struct EmitArgs {
  const ViewParams* views;
  const unsigned long long* tet_key_sorted;  // count << 40 | view << 32 | ~depth, sorted
  const uint32_t* tet_val_sorted;            // item index i (its per-view record and projections)
  const uint32_t* vis_cnt;
  const float4* vis_proj;
  const uint32_t* n_vis_ptr;
  const unsigned long long* group_off;       // from emit_scan_kernel
  uint32_t* pair_key;   // global tile id
  uint32_t* pair_val;   // item index of the (view, tet) entry
  unsigned long long cap;
  Counters* counters;
};

// 256 sorted entries per block, one per thread: the block's pair offset comes
// from emit_scan_kernel (blocks never wait on each other) plus a block-local
// scan of the entries' tile counts.  Each warp then spreads its entries'
// (entry, tile row) tasks over its lanes through a prefix of the row counts,
// so a lane whose entry spans many tile rows does not hold up the others.  A
// row's first pair slot is the entry's pairs of the rows before it: a scan of
// the row widths within the round plus the entry's pairs of earlier rounds.
// The pairs are exactly the per-entry loop's: rows in order, tiles in order,
// the first cnt of them (cnt from the projection's count), and sentinels for
// the slots an entry leaves unfilled.
__global__ void __launch_bounds__(256) emit_kernel(EmitArgs a) {
  __shared__ unsigned long long s_wsum[8];
  const uint32_t blk = blockIdx.x;
  const uint32_t n = *a.n_vis_ptr;
  if ((unsigned long long)blk * 256ull >= n) return;
  const uint32_t k = blk * 256u + threadIdx.x;
  const bool in = k < n;
  unsigned long long key = 0ull;
  uint32_t j = 0, cnt = 0;
  if (in) {
    key = a.tet_key_sorted[k];
    j = a.tet_val_sorted[k];
    cnt = key_count(key, j, a.vis_cnt);
  }
  // block exclusive scan of cnt (64-bit)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_wsum[warp] = x;
  __syncthreads();
  unsigned long long woff = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w)
    if (w < warp) woff += s_wsum[w];
  const unsigned long long off = a.group_off[blk] + woff + x - cnt;

  // this lane's entry: projected vertices and tile box
  const uint32_t view = (uint32_t)(key >> 32) & 0xFFu;
  float px[4] = {0.f, 0.f, 0.f, 0.f}, py[4] = {0.f, 0.f, 0.f, 0.f};
  TileBox tb = {0u, 0u, 0u, 0u};
  uint32_t TS = 1u, tile_base = 0u, tiles_x = 0u;
  int nrows = 0;
  if (in && cnt > 0) {
    const ViewParams& V = a.views[view];
    TS = (uint32_t)V.TS;
    tile_base = V.tile_base;
    tiles_x = (uint32_t)V.tiles_x;
    const float4 q0 = a.vis_proj[2 * (size_t)j], q1 = a.vis_proj[2 * (size_t)j + 1];
    px[0] = q0.x; px[1] = q0.z; px[2] = q1.x; px[3] = q1.z;
    py[0] = q0.y; py[1] = q0.w; py[2] = q1.y; py[3] = q1.w;
    if (tile_range(px, py, V.Wf, V.Hf, TS, tb)) nrows = (int)(tb.max_y - tb.min_y) + 1;
  }
  int pre = nrows;  // inclusive prefix of the row counts over the warp's lanes
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += y;
  }
  const int excl = pre - nrows;
  const int total = __shfl_sync(0xffffffffu, pre, 31);
  uint32_t emitted = 0u;  // pairs of this lane's entry in the rows handled so far
  bool overflow = false;
  for (int t0 = 0; t0 < total; t0 += 32) {  // warp-uniform trip count
    const int t = t0 + lane;
    int e = 0;  // the lane whose entry owns task t: first inclusive prefix > t
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
      const int pv = __shfl_sync(0xffffffffu, pre, e + st - 1);
      if (pv <= t) e += st;
    }
    const int e_excl = __shfl_sync(0xffffffffu, excl, e);
    float qx[4], qy[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      qx[q] = __shfl_sync(0xffffffffu, px[q], e);
      qy[q] = __shfl_sync(0xffffffffu, py[q], e);
    }
    TileBox eb;
    eb.min_x = __shfl_sync(0xffffffffu, tb.min_x, e);
    eb.max_x = __shfl_sync(0xffffffffu, tb.max_x, e);
    eb.min_y = __shfl_sync(0xffffffffu, tb.min_y, e);
    eb.max_y = __shfl_sync(0xffffffffu, tb.max_y, e);
    const uint32_t e_ts = __shfl_sync(0xffffffffu, TS, e);
    const uint32_t ty = eb.min_y + (uint32_t)(t - e_excl);
    uint32_t tx0 = 0u, tx1 = 0u, width = 0u;
    if (t < total && tile_row_span(qx, qy, e_ts, eb, ty, tx0, tx1)) width = tx1 - tx0 + 1u;
    uint32_t incl = width;  // inclusive scan of the row widths over the round
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t exw = incl - width;
    // the entry's first slot of this row: its pairs of earlier rounds plus the
    // widths of its earlier rows in this round
    const int first_lane = max(e_excl - t0, 0);
    const uint32_t pos = __shfl_sync(0xffffffffu, emitted, e) + exw - __shfl_sync(0xffffffffu, exw, first_lane);
    const unsigned long long e_off = __shfl_sync(0xffffffffu, off, e);
    const uint32_t e_cnt = __shfl_sync(0xffffffffu, cnt, e);
    const uint32_t e_j = __shfl_sync(0xffffffffu, j, e);
    const uint32_t e_base = __shfl_sync(0xffffffffu, tile_base, e);
    const uint32_t e_tx = __shfl_sync(0xffffffffu, tiles_x, e);
    for (uint32_t i = 0; i < width && pos + i < e_cnt; ++i) {
      const unsigned long long w = e_off + pos + i;
      if (w < a.cap) {
        a.pair_key[w] = e_base + ty * e_tx + tx0 + i;
        a.pair_val[w] = e_j;
      } else {
        overflow = true;
      }
    }
    // this lane's entry: add the widths of its rows in this round
    const int my_first = max(excl - t0, 0), my_last = min(pre - t0, 32) - 1;
    const uint32_t hi_sum = __shfl_sync(0xffffffffu, incl, max(my_last, 0));
    const uint32_t lo_sum = __shfl_sync(0xffffffffu, exw, min(my_first, 31));
    if (nrows > 0 && my_first <= my_last) emitted += hi_sum - lo_sum;
  }
  if (in && cnt > 0) {
    if (emitted < cnt) atomicOr(&a.counters->shortfall[view], 1u);
    for (uint32_t l = emitted; l < cnt; ++l) {
      const unsigned long long w = off + l;
      if (w < a.cap) {
        a.pair_key[w] = kSentinel;
        a.pair_val[w] = 0u;
      } else {
        overflow = true;
      }
    }
  }
  if (overflow) atomicOr(&a.counters->err, kErrPairOverflow);
}

// Sets *bad when an index is not below n_verts (reads only the index array):
// rmesh_create runs it before any kernel gathers through the indices.
__global__ void __launch_bounds__(256) index_range_kernel(const uint32_t* __restrict__ idx, uint64_t n,
                                                          uint32_t n_verts, uint32_t* bad) {
  bool any = false;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    any = any || idx[i] >= n_verts;
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

// Longest-first tile order for the persistent tile kernel: a tile's cost
// grows with its list length, and a long list taken last leaves the other
// CTAs idle, so tiles are bucketed by floor(log2(length)) and the buckets are
// handed out from the longest down (order within a bucket is arbitrary; every
// tile's result is independent of the order).
constexpr int kOrderBuckets = 33;  // 0: empty list; 1 + floor(log2(length)) otherwise
__device__ __forceinline__ int order_bucket(uint2 r) {
  const uint32_t len = r.y > r.x ? r.y - r.x : 0u;
  return len ? 32 - __clz(len) : 0;
}

__global__ void __launch_bounds__(256) tile_order_hist_kernel(const uint2* __restrict__ ranges, uint32_t n_tiles,
                                                              uint32_t* hist) {
  __shared__ uint32_t sh[kOrderBuckets];
  for (int i = threadIdx.x; i < kOrderBuckets; i += blockDim.x) sh[i] = 0u;
  __syncthreads();
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_tiles; t += gridDim.x * blockDim.x)
    atomicAdd(&sh[order_bucket(ranges[t])], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < kOrderBuckets; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// order[pos] = tile, bucket by bucket from the longest lists down, and inside
// a bucket in tile order (a stable counting sort by bucket): tiles of one view
// are numbered together, so a bucket's tiles of a view run close in time and
// share their tet records and span-cache lines in L2.  One block walks the
// tiles in chunks of kOrderThreads: each tile's rank among the chunk's tiles
// of its bucket comes from per-warp peer masks (one ballot per bucket bit)
// and a per-bucket scan over the warps.
constexpr int kOrderThreads = 1024;
__global__ void __launch_bounds__(kOrderThreads) tile_order_stable_kernel(const uint2* __restrict__ ranges,
                                                                          uint32_t n_tiles, const uint32_t* hist,
                                                                          uint32_t* order) {
  constexpr int kW = kOrderThreads / 32;
  __shared__ uint32_t cursor[kOrderBuckets];
  __shared__ uint32_t wcnt[kW][kOrderBuckets];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    uint32_t acc = 0u;
    for (int b = kOrderBuckets - 1; b >= 0; --b) {
      cursor[b] = acc;
      acc += hist[b];
    }
  }
  for (uint32_t base = 0; base < n_tiles; base += kOrderThreads) {
    for (int i = tid; i < kW * kOrderBuckets; i += kOrderThreads) (&wcnt[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t t = base + (uint32_t)tid;
    const bool live = t < n_tiles;
    const int b = live ? order_bucket(ranges[t]) : 63;  // 63: no bucket
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int bit = 0; bit < 6; ++bit) {
      const bool v = (b >> bit) & 1;
      const unsigned bb = __ballot_sync(0xffffffffu, v);
      peers &= v ? bb : ~bb;
    }
    const uint32_t rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
    if (live && lane == __ffs(peers) - 1) wcnt[warp][b] = (uint32_t)__popc(peers);
    __syncthreads();
    if (tid < kOrderBuckets) {  // exclusive scan of bucket tid over the warps
      uint32_t off = cursor[tid];
      for (int w = 0; w < kW; ++w) {
        const uint32_t c = wcnt[w][tid];
        wcnt[w][tid] = off;
        off += c;
      }
      cursor[tid] = off;
    }
    __syncthreads();
    if (live) order[wcnt[warp][b] + rank] = t;
    __syncthreads();
  }
}

// Per-tile [start, end) over the sorted pair keys.  Restates
// tile_ranges_compute.wgsl:10-45 per view: the end of a view's last non-empty
// tile is only written when the view had no sentinel slots (in the reference
// the sentinels follow that tile and the idx == count-1 rule never fires for
// it, leaving end = 0 from the clear).  ranges must be zeroed beforehand.
__global__ void __launch_bounds__(256) ranges_kernel(const uint32_t* __restrict__ keys,
                                                     const unsigned long long* n_ptr, unsigned long long cap,
                                                     uint2* __restrict__ ranges,
                                                     const ViewParams* views, int n_views,
                                                     const Counters* counters) {
  const unsigned long long n = *n_ptr < cap ? *n_ptr : cap;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t key = keys[idx];
    if (key == kSentinel) continue;
    const uint32_t prev = idx > 0 ? keys[idx - 1] : kSentinel;
    const uint32_t next = idx + 1 < n ? keys[idx + 1] : kSentinel;
    if (idx == 0 || key != prev) ranges[key].x = (uint32_t)idx;
    if (next != key) {
      const int v = view_of_tile(views, n_views, key);
      const bool last_of_view = (next == kSentinel) || view_of_tile(views, n_views, next) != v;
      if (!(last_of_view && counters->shortfall[v])) ranges[key].y = (uint32_t)(idx + 1);
    }
  }
}

// Debug view of the sorted pairs: the pair payload is the item index
// tet * n_views + view; map it back to the tet id (sentinel slots keep the
// reference's 0).
__global__ void __launch_bounds__(256) pair_tets_kernel(const uint32_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ vals, uint32_t n_views,
                                                        uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = keys[i] == kSentinel ? 0u : vals[i] / n_views;
}

}  // namespace rm
