// Onesweep LSD radix sort (8-bit digits, stable) with decoupled look-back.
//
// Replaces the reference's 3-kernel-per-pass DeviceRadixSort
// (crates/rmesh-sort/src/drs.rs:180-279, wgsl/drs_{upsweep,scan,downsweep}.wgsl):
// one histogram kernel computes the digit counts of every pass in a single
// read of the keys, then each pass is ONE kernel that ranks a 4096-key
// partition in shared memory (warp multi-split: peers of a digit found by one
// ballot per digit bit), looks back
// across earlier partitions for the per-digit global offset, and scatters
// through shared memory so the writes are digit-contiguous.
//
// Partitions are numbered by an atomic ticket, so every partition a block
// waits on was started earlier (forward progress without co-residency).
// Status words carry a device-side epoch instead of being cleared, so a
// captured CUDA graph can replay the sort without memsets.  All spins are
// bounded and raise kErrSpinTimeout instead of hanging.
#pragma once
#include "common.cuh"

namespace rm {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortKPT = 16;
constexpr int kSortPart = kSortThreads * kSortKPT;  // 4096 keys: the smallest partition (buffer sizing)
// Keys per thread by key width: 32-bit keys take 24 (6144-key partitions, a
// third fewer look-back steps per pass); 64-bit keys stay at 16, where 24
// would push the kernel past its register budget for two blocks per SM.
template <typename K>
struct SortCfg {
  static constexpr int KPT = sizeof(K) == 4 ? 24 : 16;
  static constexpr int PART = kSortThreads * KPT;
};
constexpr int kMaxPasses = 8;

struct SortState {
  uint32_t epoch;                       // bumped once per sort
  uint32_t ticket[kMaxPasses];          // partition tickets, reset by sort_scan_kernel
  uint32_t hist[kMaxPasses][256];       // global digit counts (zeroed by a memset per sort)
  uint32_t offs[kMaxPasses][256];       // exclusive digit offsets
};

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift) {
  return (uint32_t)(key >> shift) & 0xFFu;
}

// One read of the keys; counts digits of all passes.
template <typename K>
__global__ void __launch_bounds__(256) sort_hist_kernel(const K* __restrict__ keys, const void* n_ptr, int n_is_u64,
                                                        unsigned long long cap, int begin_bit, int passes,
                                                        SortState* st) {
  __shared__ uint32_t h[kMaxPasses][256];
  for (int i = threadIdx.x; i < kMaxPasses * 256; i += blockDim.x) (&h[0][0])[i] = 0u;
  __syncthreads();
  unsigned long long n = n_is_u64 ? *(const unsigned long long*)n_ptr : *(const uint32_t*)n_ptr;
  if (n > cap) n = cap;  // an overflowed count never reads past the buffers
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const K k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][digit_of(k, begin_bit + 8 * p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(&st->hist[0][0] + i, c);
  }
}

// Exclusive scan of each pass's 256 digit counts; bumps the epoch; resets tickets.
__global__ void sort_scan_kernel(int passes, SortState* st) {
  __shared__ uint32_t s[256];
  const int d = threadIdx.x;  // 256 threads
  for (int p = 0; p < passes; ++p) {
    s[d] = st->hist[p][d];
    __syncthreads();
    // Hillis-Steele inclusive scan
    for (int o = 1; o < 256; o <<= 1) {
      const uint32_t v = d >= o ? s[d - o] : 0u;
      __syncthreads();
      s[d] += v;
      __syncthreads();
    }
    st->offs[p][d] = s[d] - st->hist[p][d];
    __syncthreads();
  }
  if (d < kMaxPasses) st->ticket[d] = 0u;
  if (d == 0) st->epoch = st->epoch + 1u;
}

// Status word: [63:32] epoch, [31:30] flag (1 aggregate, 2 inclusive), [29:0] count.
__device__ __forceinline__ unsigned long long pack_status(uint32_t epoch, uint32_t flag, uint32_t v) {
  return ((unsigned long long)epoch << 32) | ((unsigned long long)flag << 30) | (unsigned long long)(v & 0x3FFFFFFFu);
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) onesweep_kernel(const K* __restrict__ keys_in,
                                                                const uint32_t* __restrict__ vals_in,
                                                                K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                                const void* n_ptr, int n_is_u64,
                                                                unsigned long long cap, int shift, int pass,
                                                                SortState* st, unsigned long long* status,
                                                                uint32_t* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  K* s_keys = reinterpret_cast<K*>(smem);
  uint32_t* s_vals = reinterpret_cast<uint32_t*>(smem + sizeof(K) * SortCfg<K>::PART);
  uint32_t* s_whist = s_vals + SortCfg<K>::PART;            // [kSortWarps][256]
  uint32_t* s_dstart = s_whist + kSortWarps * 256;   // [256] digit start inside the partition
  uint32_t* s_gbase = s_dstart + 256;                // [256] global base per digit
  __shared__ uint32_t s_part;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_part = atomicAdd(&st->ticket[pass], 1u);
  __syncthreads();
  const uint32_t part = s_part;
  unsigned long long n = n_is_u64 ? *(const unsigned long long*)n_ptr : *(const uint32_t*)n_ptr;
  if (n > cap) n = cap;
  const unsigned long long base = (unsigned long long)part * SortCfg<K>::PART;
  if (base >= n) return;
  const uint32_t epoch = st->epoch * (uint32_t)kMaxPasses + (uint32_t)pass;  // unique per (sort, pass)

  // warp-striped load: warp w owns keys [w*32*KPT, (w+1)*32*KPT), lane-minor
  K k[SortCfg<K>::KPT];
  uint32_t v[SortCfg<K>::KPT];
  const unsigned long long wbase = base + (unsigned long long)warp * 32 * SortCfg<K>::KPT;
#pragma unroll
  for (int i = 0; i < SortCfg<K>::KPT; ++i) {
    const unsigned long long idx = wbase + (unsigned long long)i * 32 + lane;
    if (idx < n) {
      k[i] = keys_in[idx];
      v[i] = vals_in[idx];
    } else {
      k[i] = ~(K)0;  // digit 0xFF, ranked after every real key of this partition
      v[i] = 0u;
    }
  }
  for (int i = lane; i < 256; i += 32) s_whist[warp * 256 + i] = 0u;
  __syncwarp();

  // warp multi-split: rank of each key among equal digits of this warp, in order
  uint32_t rank[SortCfg<K>::KPT];
  const unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < SortCfg<K>::KPT; ++i) {
    const uint32_t d = digit_of(k[i], shift);
    // lanes holding the same digit: one ballot per digit bit
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const bool bit = (d >> b) & 1u;
      const unsigned bb = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bb : ~bb;
    }
    const int leader = __ffs(peers) - 1;
    // the leader advances the warp's digit counter; the shuffle that hands the
    // old count to its peers also orders this key's update before the next
    // key's (whose leader may be another lane)
    uint32_t old = 0u;
    if (lane == leader) old = atomicAdd(&s_whist[warp * 256 + d], (uint32_t)__popc(peers));
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[i] = old + __popc(peers & lt_mask);
  }
  __syncthreads();

  // per digit: exclusive prefix across warps; partition count
  const uint32_t d = (uint32_t)tid;  // 256 threads == 256 digits
  uint32_t cnt = 0u;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const uint32_t c = s_whist[w * 256 + d];
    s_whist[w * 256 + d] = cnt;
    cnt += c;
  }
  // keys past n were counted in digit 0xFF; they sit after all real keys and are dropped below
  // publish aggregate, look back for the exclusive prefix of this digit
  unsigned long long* my = status + (unsigned long long)part * 256 + d;
  uint32_t prefix = 0u;
  if (part == 0) {
    st_volatile_u64(my, pack_status(epoch, 2u, cnt));
  } else {
    st_volatile_u64(my, pack_status(epoch, 1u, cnt));
    int64_t p = (int64_t)part - 1;
    uint32_t spins = 0;
    while (p >= 0) {
      const unsigned long long s = ld_volatile_u64(status + (unsigned long long)p * 256 + d);
      const uint32_t e = (uint32_t)(s >> 32), flag = (uint32_t)(s >> 30) & 3u;
      if (e != epoch || flag == 0u) {
        if (++spins > kSpinLimit) {
          atomicOr(err, kErrSpinTimeout);
          break;
        }
        __nanosleep(20);
        continue;
      }
      prefix += (uint32_t)(s & 0x3FFFFFFFu);
      if (flag == 2u) break;
      --p;
    }
    __threadfence();
    st_volatile_u64(my, pack_status(epoch, 2u, prefix + cnt));
  }
  s_gbase[d] = st->offs[pass][d] + prefix;

  // block exclusive scan of cnt over digits -> start of each digit inside the partition
  s_dstart[d] = cnt;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const uint32_t t = d >= (uint32_t)o ? s_dstart[d - o] : 0u;
    __syncthreads();
    s_dstart[d] += t;
    __syncthreads();
  }
  const uint32_t incl = s_dstart[d];
  __syncthreads();
  s_dstart[d] = incl - cnt;
  __syncthreads();

  // scatter into shared memory in sorted order
#pragma unroll
  for (int i = 0; i < SortCfg<K>::KPT; ++i) {
    const uint32_t dg = digit_of(k[i], shift);
    const uint32_t pos = s_dstart[dg] + s_whist[warp * 256 + dg] + rank[i];
    s_keys[pos] = k[i];
    s_vals[pos] = v[i];
  }
  __syncthreads();

  // write out; consecutive threads write consecutive slots of one digit run
  for (int j = tid; j < SortCfg<K>::PART; j += kSortThreads) {
    const K kk = s_keys[j];
    const uint32_t dg = digit_of(kk, shift);
    const unsigned long long out = (unsigned long long)s_gbase[dg] + (unsigned long long)(j - s_dstart[dg]);
    if (out < n) {
      keys_out[out] = kk;
      vals_out[out] = s_vals[j];
    }
  }
}

}  // namespace rm
