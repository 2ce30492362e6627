// Tiled compositing: forward, adjoint, and the fused forward+loss+adjoint.
//
// Reference kernels restated:
//   forward   crates/rmesh-render/src/wgsl/rasterize_compute.wgsl:92-511
//   loss      crates/rmesh-train/src/wgsl/loss_compute.wgsl:24-72
//   adjoint   crates/rmesh-backward/src/wgsl/backward_tiled_compute.wgsl:154-587
//
// B200 layout.  One CTA per tile (or a persistent CTA pulling tiles from a
// queue), one thread owning each pixel's compositing state in registers, and
// the tile's tets processed in batches of kBatch = 32:
//
//   stage    warp 0 stages the batch's 144-byte per-view tet records (face
//            planes, colour base, projected vertices; written once per
//            (view, tet) by the project kernel) into shared memory with TMA
//            bulk copies (double buffered: batch b+1 is in flight while batch
//            b is composited), and with them each pair's span record of the
//            pass (pair_spans_kernel, below: every tile row's pixel span under
//            the reference scanline's rule and the pixels of the rows above);
//   spans    every covered (pixel, tet) pair is an "item", numbered tet-major
//            through the records' row offsets and one scan over the batch's
//            tets, and each pixel gets a 32-bit mask of the tets covering it;
//   phase 0  item-parallel (every thread busy): ray-tet intersection and the
//            segment integral of each item -> premultiplied colour, depth;
//   phase 1  pixel-sequential (the only order-dependent part, a few
//            instructions per item): the pixel's owner walks its mask and
//            composites front to back (forward) or undoes back to front and
//            records the restored transmittance and d(logT) (adjoint);
//   phase 2  adjoint only, item-parallel: the gradient of each item, summed
//            per thread over a run of one tet's items, then a warp-segmented
//            reduction by tet (a tet's runs sit in adjacent lanes) into 24
//            shared moments per tet, from which the tet's 19 gradients are
//            rebuilt and flushed to global memory with five 16-byte vector
//            atomics per tet and batch.
// A tet covers ~5-20 of a tile's 144-256 pixels, so working on items keeps
// all lanes busy where a thread-per-pixel sweep would idle most of them.
// Batches whose item count exceeds the item buffer run in several sub-batches.
//
// Semantics kept from the reference: the forward includes vertices inside a
// pixel row (rasterize_compute.wgsl:236-242) and skips pixels whose
// log-transmittance fell below -13.8 (:257-262, :338); the adjoint uses edge
// crossings only (backward_tiled_compute.wgsl:241-299), takes the ray origin at
// the camera, undoes every covered tet (clamping log T at 0) and skips the
// gradient when the restored transmittance is below 1e-6 (:424-437).
#pragma once
#include "common.cuh"
#include "project.cuh"
#include "tma.cuh"

namespace rm {

constexpr int kBatch = 32;
// Adjoint span cache rows per tet (tile rows, padded to 16: a tet's cached rows
// are one 16-byte line).  A row's span [lo, hi] (columns < 16) is one byte,
// lo << 4 | hi; an empty row is 0xF0 (lo > hi).
constexpr int kSpanRows = 16;
// per-pair span record of one rule: kSpanRows span bytes, then kSpanRows
// bytes holding the pair's covered pixels in the rows above each row
constexpr int kSpanRec = 2 * kSpanRows;
__device__ __forceinline__ uint8_t pack_span(short2 sp) {
  return sp.x > sp.y ? (uint8_t)0xF0u : (uint8_t)((sp.x << 4) | sp.y);
}
__device__ __forceinline__ short2 unpack_span(uint8_t v) {
  const int lo = v >> 4, hi = v & 15;
  return lo > hi ? make_short2(0, -1) : make_short2((short)lo, (short)hi);
}
constexpr int kMom = 24;      // adjoint moments per tet (see phase 2)
constexpr int kMomHalf = 12;  // moments transposed per reduction pass
// per-lane row of the warp's reduction buffer: 16 face sums (face f at 4f..4f+3)
// and the tet slot at column 16; odd stride, so lanes hit distinct banks
constexpr int kRedCols = 17;

enum TileMode : int { kModeForward = 0, kModeBackward = 1, kModeTrain = 2, kModeError = 3 };

struct TileArgs {
  const ViewParams* views;
  int n_views;
  uint32_t n_tiles;
  const uint2* ranges;
  const uint32_t* pair_val;    // index of the pair's per-view tet record
  const TetView* vis_view;     // per-(view, visible tet) records
  const TetRec* rec;           // tet records (vertex positions for the gradient flush)
  const float4* color4;
  uint32_t color_view_stride;  // 0: colours shared by all views; M: per-view colours
  float* rgba;                 // [pixels][4] (forward output; optional in train mode)
  float* aux;                  // [pixels][8 + aux_dim] (optional, forward only)
  const float* aux_data;       // [M][aux_dim] per-tet custom channels (aux_dim > 0)
  int aux_dim;
  const float* dl_rgba;        // [pixels][4] (backward mode)
  // backward mode with AUX: gradient of the custom aux channels [pixels][aux_dim]
  // and the per-tet aux data gradient [M][aux_dim] (accumulated)
  const float* dl_aux;
  float* d_aux;
  const float* gt_rgb;         // [pixels][3] (train mode)
  const float* pixel_err;      // [pixels] (error mode)
  const float* ssim_err;       // [pixels] (error mode)
  float* tet_err;              // [M][16] (error mode, accumulated)
  int* tet_count;              // [M][2] (error mode, accumulated)
  float* grad_slot;            // [M][kGradSlot]
  // SH colours: per-entry colours (the min_t path reads them) and per-entry
  // colour gradients, which then go through the SH adjoint instead of the
  // base-colour slot
  const float4* vis_color;
  float4* vis_dcolor;
  Counters* counters;
  const AdamParams* hp;
  int persistent;
  // per sorted pair position: the pair's span record under the forward's rule
  // and under the adjoint's (kSpanRec bytes each: one-byte row spans, see
  // pack_span, and the pixels of the rows above each row), from pair_spans_kernel
  const uint8_t* spans_fwd;
  const uint8_t* spans_adj;
  // persistent launches: ticket -> tile (longest lists first); nullptr = identity
  const uint32_t* tile_order;
  // the launch covers global tiles [tile_lo, tile_lo + n_tiles) (the views of
  // one tile configuration); tile_order holds indices relative to tile_lo
  uint32_t tile_lo;
  uint32_t* ticket;  // persistent tile-queue head of this launch (zeroed before it)
};

// Launch shape of a tile size.  WIDE doubles the threads per tile: the pixel
// phases use the first TS*TS threads, the item-parallel phases all of them,
// with larger sub-batches and half the resident CTAs.
template <int TS, bool AUX, bool WIDE = false>
struct TileCfg {
  static constexpr int NT = (WIDE ? 2 : 1) * (((TS * TS + 31) / 32) * 32);
  static constexpr int NW = NT / 32;
  // items per sub-batch; 920 for 12x12 tiles fills a quarter of the SM's
  // 228 KB of shared memory (four resident CTAs, the register limit at 96
  // registers per thread): fewer sub-batches, fewer block barriers
  static constexpr int CAP = WIDE ? (TS == 8 ? 512 : (TS == 12 ? 2048 : 1024)) : (TS == 12 ? 920 : 512);
  // resident CTAs per SM the register budget is sized for
  static constexpr int MINB = (WIDE ? 1 : 2) * (TS == 16 ? 1 : (TS == 12 ? 2 : 4));
};

template <int TS, bool AUX, bool WIDE = false>
struct __align__(16) TileSmem {
  using Cfg = TileCfg<TS, AUX, WIDE>;
  TetView view[2][kBatch];  // staged per-view tet records (double buffered)
  uint8_t span_pf[kBatch][kSpanRec];  // the next batch's span records (bulk copy)
  float mom[kBatch][kMom];  // adjoint moments per tet (phase 2)
  float4 pdir[TS * TS];     // pixel ray direction; w: the pixel's dL/dR (adjoint)
  float2 pdl[TS * TS];      // the pixel's dL/dG, dL/dB (adjoint); pixel and SSIM error (error mode)
  float4 item[Cfg::CAP];    // (cp.rgb, od) -> adjoint: (t_prev, d_od_state, has, aux_s)
  // per item: (t_min, t_max) and the packed faces | tet | pixel (pack_item);
  // its alpha_t = exp(-od) is recomputed from the od the item keeps
  float2 itemt[Cfg::CAP];
  uint32_t itemp[Cfg::CAP];
  float red[Cfg::NW][32][kRedCols];  // per-warp face sums and transpose (odd row stride)
  uint32_t toff[kBatch + 1];   // tet-major item offsets
  uint32_t pmask[TS * TS];
  uint8_t span[kBatch][TS];  // per (tet, row): the row's pixel span, packed as pack_span
  // per (tet, row): item index of the row's column 0 -- relative to the tet's
  // first item after the prefixes, to the sub-batch's first item after fill
  int16_t rowoff[kBatch][TS];
  uint16_t ipix[Cfg::CAP];  // (tet slot << 8) | pixel of each item of the sub-batch (tet-major)
  uint64_t bar[2];
  float lsum[16];
  uint32_t tile;
};

// Pixel of thread tid: 8x4 pixel blocks per warp for 16x16 tiles, row-major
// otherwise.  Threads past TS*TS (12x12 tiles use 160 threads, and the wide
// configurations twice the pixel count) get a real pixel's coordinates but are
// marked out of tile.
template <int TS>
__device__ __forceinline__ void pixel_of_thread(int tid, int& row, int& col, bool& in_tile) {
  if (TS == 16) {
    const int t = tid & 255;
    const int w = t >> 5, l = t & 31;
    col = (w & 1) * 8 + (l & 7);
    row = (w >> 1) * 4 + (l >> 3);
    in_tile = tid < 256;
  } else {
    in_tile = tid < TS * TS;
    const int t = in_tile ? tid : TS * TS - 1;
    row = t / TS;
    col = t - (t / TS) * TS;
  }
}

__device__ __forceinline__ float4 rec_vertex(const TetRec& r, int i) {
  return i == 0 ? r.a : (i == 1 ? r.b : (i == 2 ? r.c : r.d));
}
__device__ __forceinline__ bool face_flipped(const TetView& tv, int f) {
  return (__float_as_uint(tv.gm.w) >> f) & 1u;
}

// Ray vs the four inward face planes with the reference's rules
// (rasterize_compute.wgsl:355-390): |den| < 1e-20 is parallel (outside if
// num > 0), entry = max t over den > 0 (strict), exit = min t over den < 0.
// Exact arithmetic: t_max - t_min cancels for thin tets.
__device__ __forceinline__ bool intersect4(const float4* nrm, const float* num_override, float dx, float dy, float dz,
                                           float& t_min, float& t_max, int& fmin, int& fmax) {
  t_min = -3.402823e38f;
  t_max = 3.402823e38f;
  fmin = 0;
  fmax = 0;
  bool ok = true;
  int entry = 4;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float4 n = nrm[f];
    const float den = dot3x(n.x, n.y, n.z, dx, dy, dz);
    const float num = num_override ? num_override[f] : n.w;
    if (fabsf(den) < 1e-20f) {
      if (num > 0.0f) ok = false;
      continue;
    }
    const float t = fdv(num, den);
    if (den > 0.0f) {
      if (t > t_min) { t_min = t; fmin = f; entry = f; }
    } else {
      if (t < t_max) { t_max = t; fmax = f; }
    }
  }
  if (entry == 4) fmin = 4;  // no entering face (the forward's entry normal is then zero)
  return ok && t_min < t_max;
}

// Segment integral of one item (rasterize_compute.wgsl:394-410).
struct Integral {
  float csr, csg, csb, cer, ceg, ceb;  // ReLU'd colours at entry / exit
  float csr_r, csg_r, csb_r, cer_r, ceg_r, ceb_r;
  float dist, od_raw, od, alpha_t, ph, w0, w1;
};
__device__ __forceinline__ void integrate(const float4& cb, float dcdt, float t_min, float t_max, Integral& I,
                                          float alpha_known = -1.0f) {
  I.csr_r = cb.x + dcdt * t_min; I.csg_r = cb.y + dcdt * t_min; I.csb_r = cb.z + dcdt * t_min;
  I.cer_r = cb.x + dcdt * t_max; I.ceg_r = cb.y + dcdt * t_max; I.ceb_r = cb.z + dcdt * t_max;
  I.csr = fmaxf(I.csr_r, 0.f); I.csg = fmaxf(I.csg_r, 0.f); I.csb = fmaxf(I.csb_r, 0.f);
  I.cer = fmaxf(I.cer_r, 0.f); I.ceg = fmaxf(I.ceg_r, 0.f); I.ceb = fmaxf(I.ceb_r, 0.f);
  I.dist = t_max - t_min;
  I.od_raw = cb.w * I.dist;
  I.od = clipf(I.od_raw, 1e-8f, 88.0f);
  I.alpha_t = alpha_known >= 0.0f ? alpha_known : __expf(-I.od);
  I.ph = fabsf(I.od) < 0.02f ? 1.0f + I.od * (-0.5f + I.od * (1.0f / 6.0f + I.od * (-1.0f / 24.0f)))
                             : clipf(__fdividef(1.0f - I.alpha_t, I.od), kMinVal, kMaxVal);
  I.w0 = I.ph - I.alpha_t;
  I.w1 = 1.0f - I.ph;
}

// Pixel spans of tile row `row` of one (tile, tet) pair, packed as pack_span:
// fwd under the forward's rule (rasterize_compute.wgsl:170-275: a row is
// reached when an edge crosses its centre line or a vertex lies in the row),
// adj under the adjoint's (backward_tiled_compute.wgsl:241-299: edge crossings
// only).  The vertex projections are taken minus the tile origin; columns past
// valid_cols (outside the image) are dropped, as the reference skips their
// pixels (rasterize_compute.wgsl:332).  The projections use fast arithmetic,
// and spans include pixels up to 0.001 px outside the silhouette, where the
// exact ray test misses anyway, so a last-bit difference in a span end changes
// no pixel value.
__device__ __forceinline__ short2 span_of_cols(float xl, float xr, int valid_cols) {
  short2 sp = make_short2(0, -1);
  if (xl <= xr) {
    // directed-rounding conversions: ceil / floor and the conversion in one step
    const int32_t lo = max(__float2int_ru(xl - 0.5f - 0.001f), 0);
    const int32_t hi = min(__float2int_rd(xr - 0.5f + 0.001f), valid_cols - 1);
    if (lo <= hi) sp = make_short2((short)lo, (short)hi);
  }
  return sp;
}
// sx, sy: the four vertices sorted by y.  An edge crosses the row's centre
// line yc when its lower end is <= yc < its upper end, so with b vertices at
// or below yc the crossing edges are exactly the pairs (i, j) of sorted ranks
// i < b <= j: three edges for b = 1 or 3, four for b = 2, none otherwise.
__device__ __forceinline__ void row_spans(const float sx[4], const float sy[4], int row, int valid_cols, uint8_t& fwd,
                                          uint8_t& adj) {
  fwd = 0xF0u;
  adj = 0xF0u;
  const float yc = fa((float)row, 0.5f);
  const float blo = fs(yc, 0.5f), bhi = fa(yc, 0.5f);
  // the adjoint's reach (some edge crosses yc) implies the forward's
  if (!(sy[3] >= blo && sy[0] < bhi)) return;
  const int nb = (sy[0] <= yc ? 1 : 0) + (sy[1] <= yc ? 1 : 0) + (sy[2] <= yc ? 1 : 0) + (sy[3] <= yc ? 1 : 0);
  float xl = 1e10f, xr = -1e10f;
  auto cross = [&](float xi, float yi, float xj, float yj) {
    const float t = __fdividef(yc - yi, yj - yi);
    const float x = xi + t * (xj - xi);
    xl = fminf(xl, x);
    xr = fmaxf(xr, x);
  };
  if (nb >= 1 && nb <= 3) {
    cross(sx[0], sy[0], sx[3], sy[3]);  // (0, 3) crosses in every band
    // (0, 1) | (0, 2) | (1, 3) for b = 1 | 2 | 3
    const float ax = nb == 3 ? sx[1] : sx[0], ay = nb == 3 ? sy[1] : sy[0];
    const float bx = nb == 1 ? sx[1] : (nb == 2 ? sx[2] : sx[3]), by = nb == 1 ? sy[1] : (nb == 2 ? sy[2] : sy[3]);
    cross(ax, ay, bx, by);
    // (0, 2) | (1, 2) | (2, 3)
    const float cx = nb == 1 ? sx[0] : (nb == 2 ? sx[1] : sx[2]), cy = nb == 1 ? sy[0] : (nb == 2 ? sy[1] : sy[2]);
    const float dx = nb == 3 ? sx[3] : sx[2], dy = nb == 3 ? sy[3] : sy[2];
    cross(cx, cy, dx, dy);
    if (nb == 2) cross(sx[1], sy[1], sx[3], sy[3]);  // (1, 3)
  }
  adj = pack_span(span_of_cols(xl, xr, valid_cols));  // empty when no edge crosses yc
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float vyq = sy[q];
    if (vyq >= blo && vyq < bhi) {
      xl = fminf(xl, sx[q]);
      xr = fmaxf(xr, sx[q]);
    }
  }
  fwd = pack_span(span_of_cols(xl, xr, valid_cols));
}

// itemp packs the adjoint's exit/entry faces, the tet's batch slot and the pixel
__device__ __forceinline__ uint32_t pack_item(int fmin, int fmax, int k, int p) {
  return (uint32_t)fmin | ((uint32_t)fmax << 3) | ((uint32_t)k << 5) | ((uint32_t)p << 10);
}

template <int TS, int MODE, bool AUX, bool WIDE>
__global__ void __launch_bounds__(TileCfg<TS, AUX, WIDE>::NT, TileCfg<TS, AUX, WIDE>::MINB) tile_kernel(TileArgs a) {
  using Cfg = TileCfg<TS, AUX, WIDE>;
  constexpr int NT = Cfg::NT;
  constexpr int NW = Cfg::NW;
  constexpr int CAP = Cfg::CAP;
  extern __shared__ __align__(16) unsigned char tile_smem_raw[];
  TileSmem<TS, AUX, WIDE>& s = *reinterpret_cast<TileSmem<TS, AUX, WIDE>*>(tile_smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int prow, pcol;
  bool in_tile;
  pixel_of_thread<TS>(tid, prow, pcol, in_tile);
  const int pl = prow * TS + pcol;

  if (tid == 0) {
    mbar_init(&s.bar[0], 1);
    mbar_init(&s.bar[1], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < kBatch * kMom; i += NT) (&s.mom[0][0])[i] = 0.0f;
  __syncthreads();
  uint32_t phase_bits = 0u;  // parity of the next phase of bar[0] (bit 0) and bar[1] (bit 1)
  bool failed = false;

  const uint32_t first_tile = blockIdx.x;
  while (true) {
    if (tid == 0) {
      uint32_t t = first_tile;
      if (a.persistent) {
        t = atomicAdd(a.ticket, 1u);
        if (a.tile_order && t < a.n_tiles) t = a.tile_order[t];
        else if (t >= a.n_tiles) t = 0xFFFFFFFFu;
      }
      s.tile = t;
    }
    __syncthreads();
    if (s.tile >= a.n_tiles || failed) break;
    const uint32_t g = s.tile + a.tile_lo;  // global tile id
    const int view = view_of_tile(a.views, a.n_views, g);
    const ViewParams& V = a.views[view];
    const uint32_t local_tile = g - V.tile_base;
    const uint32_t tile_y = local_tile / (uint32_t)V.tiles_x;
    const uint32_t tile_x = local_tile - tile_y * (uint32_t)V.tiles_x;
    const float tile_ox = (float)(tile_x * (uint32_t)TS), tile_oy = (float)(tile_y * (uint32_t)TS);
    const uint32_t px = tile_x * (uint32_t)TS + (uint32_t)pcol;
    const uint32_t py = tile_y * (uint32_t)TS + (uint32_t)prow;
    const bool valid = in_tile && px < (uint32_t)V.W && py < (uint32_t)V.H;
    const size_t pix = (size_t)V.pix_base + (size_t)py * (size_t)V.W + px;
    const uint2 range = a.ranges[g];
    const uint32_t rs = range.x, re = range.y;
    // pixels of this tile inside the image
    const int valid_rows = min(TS, V.H - (int)(tile_y * TS));

    // pixel ray (rasterize_compute.wgsl:343-349), explicitly rounded: the ray and
    // the plane hits feed t_max - t_min, which cancels for thin tets, so they
    // are evaluated exactly as the reference's left-to-right float math.
    float dx, dy, dz;
    {
      float ux = fdv(fs(fa((float)px, 0.5f), V.cx), V.fx);
      float uy = fdv(fs(fa((float)py, 0.5f), V.cy), V.fy);
      float uz = 1.0f;
      float l = __fsqrt_rn(dot3x(ux, uy, uz, ux, uy, uz));
      ux = fdv(ux, l); uy = fdv(uy, l); uz = fdv(uz, l);
      const float wx = fa(fa(fm(V.c2w[0], ux), fm(V.c2w[3], uy)), fm(V.c2w[6], uz));
      const float wy = fa(fa(fm(V.c2w[1], ux), fm(V.c2w[4], uy)), fm(V.c2w[7], uz));
      const float wz = fa(fa(fm(V.c2w[2], ux), fm(V.c2w[5], uy)), fm(V.c2w[8], uz));
      l = __fsqrt_rn(dot3x(wx, wy, wz, wx, wy, wz));
      dx = fdv(wx, l); dy = fdv(wy, l); dz = fdv(wz, l);
    }
    if (in_tile) s.pdir[pl] = make_float4(dx, dy, dz, 0.0f);
    const float camx = V.cam[0], camy = V.cam[1], camz = V.cam[2];
    // forward ray origin cam + dir * min_t (rasterize_compute.wgsl:352); the
    // adjoint keeps the origin at the camera (backward_tiled_compute.wgsl:377)
    const bool has_min_t = V.min_t != 0.0f;

    // ---------------- batch machinery ----------------
    // dir = -1: front-to-back from `first` downwards (forward); +1: upwards (adjoint)
    // Warp 0 lane l loads the record index of the batch's l-th pair one batch
    // ahead of the copy that uses it, so the load's latency overlaps a batch.
    auto load_idx = [&](uint32_t first, int nb, int dir) -> uint32_t {
      if (warp != 0 || lane >= nb) return 0u;
      return a.pair_val[dir < 0 ? first - (uint32_t)lane : first + (uint32_t)lane];
    };
    // span_src: the batch's span records (kSpanRec bytes per list position,
    // ascending), copied into span_pf on the same barrier
    auto issue = [&](int buf, int nb, uint32_t idx, const uint8_t* span_src) {
      if (warp == 0) {
        if (lane == 0) {
          fence_proxy_async_smem();
          const uint32_t span_bytes = span_src ? (uint32_t)(nb * kSpanRec) : 0u;
          mbar_arrive_expect_tx(&s.bar[buf], (uint32_t)nb * (uint32_t)sizeof(TetView) + span_bytes);
          if (span_src) bulk_copy_g2s(&s.span_pf[0][0], span_src, span_bytes, &s.bar[buf]);
        }
        __syncwarp();
        if (lane < nb)
          bulk_copy_g2s(&s.view[buf][lane], a.vis_view + idx, (uint32_t)sizeof(TetView), &s.bar[buf]);
      }
    };
    // every thread waits on the phase; the outcome is made block-uniform
    auto wait_buf = [&](int buf) {
      const bool ok = mbar_wait_bounded(&s.bar[buf], (phase_bits >> buf) & 1u, 1u << 20);
      phase_bits ^= 1u << buf;
      if (__syncthreads_or(!ok)) {
        failed = true;
        if (tid == 0) atomicOr(&a.counters->err, kErrSpinTimeout);
      }
    };
    // Row table of the batch, kept in registers by every warp: lane l < nb holds
    // tet l's first row and row count under the forward's reach rule (a row is
    // reached when an edge crosses its centre or a vertex lies in it; the
    // adjoint's rows, edge crossings only, are a subset) clipped to the image,
    // and the inclusive prefix of the counts.  Span, prefix and fill tasks are
    // (tet, reachable row) pairs numbered through this prefix, so no thread
    // works on a row the tet cannot touch.
    int rr_lo = 0, rr_n = 0, rr_pre = 0, rr_total = 0;
    auto row_ranges = [&](int buf, int nb) {
      int lo = 0, n = 0;
      if (lane < nb) {
        const TetView& tv = s.view[buf][lane];
        if (!((__float_as_uint(tv.gm.w) >> 4) & 1u)) {
          const float4 gy4 = tv.py;
          // min/max of the tile-local y (subtracting the tile origin is monotonic)
          const float ylo = fs(fminf(fminf(gy4.x, gy4.y), fminf(gy4.z, gy4.w)), tile_oy);
          const float yhi = fs(fmaxf(fmaxf(gy4.x, gy4.y), fmaxf(gy4.z, gy4.w)), tile_oy);
          // row r is reached iff yhi >= r and ylo < r + 1, i.e. floor(ylo) <= r <= floor(yhi)
          const float flo = fmaxf(floorf(ylo), 0.0f);
          const float fhi = fminf(floorf(yhi), (float)(valid_rows - 1));
          if (flo <= fhi) {
            lo = (int)flo;
            n = (int)fhi - lo + 1;
          }
        }
      }
      int x = n;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      rr_lo = lo;
      rr_n = n;
      rr_pre = x;
      rr_total = __shfl_sync(0xffffffffu, x, 31);
    };
    // tet of task t: the first tet whose inclusive prefix exceeds t (all lanes call)
    auto task_tet = [&](int t) -> int {
      int k = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const int pv = __shfl_sync(0xffffffffu, rr_pre, k + st - 1);
        if (pv <= t) k += st;
      }
      return k;
    };
    // row of task t of tet k (all lanes call)
    auto task_row = [&](int t, int k) -> int { return __shfl_sync(0xffffffffu, rr_lo - (rr_pre - rr_n), k) + t; };
    // the batch's span records, already copied into span_pf by the batch's
    // bulk copy (pair_spans_kernel wrote them per list position): tet k is list
    // position k of the copy, or nb - 1 - k when the batch runs front to back
    // (rev).  Each row's span goes to the span table and its item offset
    // relative to the tet's first item (the pixels of the rows above, minus the
    // row's first column) to rowoff.
    auto load_spans = [&](int buf, int nb, bool rev) {
      row_ranges(buf, nb);
      for (int i = tid; i < TS * TS; i += NT) s.pmask[i] = 0u;
      for (int task = tid; task < nb * TS; task += NT) {
        const int k = task / TS, row = task - (task / TS) * TS;
        const uint8_t* rec = s.span_pf[rev ? nb - 1 - k : k];
        const uint8_t sb = rec[row];
        s.span[k][row] = sb;
        s.rowoff[k][row] = (int16_t)((int)rec[kSpanRows + row] - (int)unpack_span(sb).x);
      }
    };
    // tet-major item offsets (warp 0, lane = tet, read from the span records in
    // span_pf, so it runs beside load_spans before the same barrier): a tet's
    // item count is its last reachable row's pixels above plus that row's width
    auto prefixes = [&](int nb, bool rev) {
      if (warp == 0) {
        uint32_t cnt = 0;
        if (lane < nb && rr_n > 0) {
          const int last = rr_lo + rr_n - 1;
          const uint8_t* rec = s.span_pf[rev ? nb - 1 - lane : lane];
          const short2 sp = unpack_span(rec[last]);
          cnt = (uint32_t)rec[kSpanRows + last] + (uint32_t)max(sp.y - sp.x + 1, 0);
        }
        uint32_t x = cnt;  // exclusive scan over the batch's tets (nb <= 32)
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (lane < nb) s.toff[lane + 1] = x;
        if (lane == 0) s.toff[0] = 0u;
      }
    };
    // item pixel ids of tets [k0, k1), numbered from the sub-batch's first
    // item, and their per-pixel coverage bits.  Only phase 0 reads the ids, so
    // the next sub-batch's are written in the tail of the current one (before
    // its closing barrier); the coverage bits of later tets are masked off there.
    auto fill = [&](int k0, int k1) {
      const uint32_t base0 = s.toff[k0];
      // tasks of tets [k0, k1) in the row table
      const int tb = __shfl_sync(0xffffffffu, rr_pre - rr_n, k0);
      const int te = k1 >= 32 ? rr_total : __shfl_sync(0xffffffffu, rr_pre - rr_n, k1);
      for (int t0 = tb + warp * 32; t0 < te; t0 += NT) {  // warp-uniform trip count
        const int t = t0 + lane;
        const int k = task_tet(t);
        const int row = task_row(t, k);
        if (t >= te) continue;
        const short2 sp = unpack_span(s.span[k][row]);
        if (sp.x > sp.y) continue;
        // rebase the row's offset onto the sub-batch (read by item_of)
        const int ro = (int)s.rowoff[k][row] + (int)(s.toff[k] - base0);
        s.rowoff[k][row] = (int16_t)ro;
        const uint32_t base = (uint32_t)(ro + sp.x);
        for (int c = sp.x; c <= sp.y; ++c) {
          s.ipix[base + (uint32_t)(c - sp.x)] = (uint16_t)((k << 8) | (row * TS + c));
          atomicOr(&s.pmask[row * TS + c], 1u << k);
        }
      }
    };
    // item gi of the sub-batch -> (tet k, pixel index in tile)
    auto decode = [&](uint32_t gi, int& k, int& p) {
      const uint32_t e = s.ipix[gi];
      k = (int)(e >> 8);
      p = (int)(e & 255u);
    };
    // item index of (tet k, this thread's pixel) inside the current sub-batch
    // (one shared load: fill rebased the row offsets onto the sub-batch)
    auto item_of = [&](int k, uint32_t) -> uint32_t { return (uint32_t)((int)s.rowoff[k][prow] + pcol); };
    // sub-batch end (>= k0 + 1): the batch's remaining items split into the
    // fewest sub-batches of at most CAP items, of about equal size, so that
    // no short remainder leaves most threads of a phase idle
    auto sub_end = [&](int k0, int nb) -> int {
      const uint32_t base = s.toff[k0];
      const uint32_t rem = s.toff[nb] - base;
      if (rem <= (uint32_t)CAP) return nb;
      const uint32_t parts = (rem + (uint32_t)CAP - 1u) / (uint32_t)CAP;
      const uint32_t target = (rem + parts - 1u) / parts;
      int k1 = k0 + 1;
      while (k1 < nb && s.toff[k1] - base < target && s.toff[k1 + 1] - base <= (uint32_t)CAP) ++k1;
      return k1;
    };
    // phase 0: item-parallel intersection + integral.  clip_lo: 0 for the
    // forward (rasterize_compute.wgsl:409), -1e20 for the adjoint (:411).
    auto phase0 = [&](int buf, int k0, int k1, bool fwd) {
      const uint32_t base = s.toff[k0];
      const uint32_t n_items = s.toff[k1] - base;
      for (uint32_t i = tid; i < n_items; i += NT) {
        int k, p;
        decode(i, k, p);
        const float4 d = s.pdir[p];
        float numo[4];
        const float* nump = nullptr;
        float bcr_o = 0.f, bcg_o = 0.f, bcb_o = 0.f;
        const TetView& tv = s.view[buf][k];
        if (fwd && has_min_t) {
          // origin cam + d*min_t: num = dot(n, va - o), base offset dot(g, o - v0)
          const float oxp = fa(camx, fm(d.x, V.min_t)), oyp = fa(camy, fm(d.y, V.min_t)),
                      ozp = fa(camz, fm(d.z, V.min_t));
          const uint32_t tet = tv.meta.x;
          const TetRec rr = a.rec[tet];
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            const float4 n = tv.nrm[f];
            const float4 v = rec_vertex(rr, kFaces[f][0]);
            numo[f] = dot3x(n.x, n.y, n.z, fs(v.x, oxp), fs(v.y, oyp), fs(v.z, ozp));
          }
          nump = numo;
          const float4 gg = tv.gm;
          const float bo = dot3x(gg.x, gg.y, gg.z, fs(oxp, rr.a.x), fs(oyp, rr.a.y), fs(ozp, rr.a.z));
          const float4 cc = a.vis_color ? a.vis_color[tv.meta.y] : a.color4[(size_t)a.color_view_stride * view + tet];
          bcr_o = fa(cc.x, bo); bcg_o = fa(cc.y, bo); bcb_o = fa(cc.z, bo);
        }
        float t_min, t_max;
        int fmin, fmax;
        float4 out = make_float4(0.f, 0.f, 0.f, -1.0f);  // od < 0: the ray misses
        float2 out_t = make_float2(0.f, 0.f);
        uint32_t out_p = 0u;
        const bool hit = intersect4(tv.nrm, nump, d.x, d.y, d.z, t_min, t_max, fmin, fmax);
        if (hit) {
          float4 cb = tv.cb;
          if (fwd && has_min_t) cb = make_float4(bcr_o, bcg_o, bcb_o, cb.w);
          const float4 gg = tv.gm;
          const float dcdt = dot3x(gg.x, gg.y, gg.z, d.x, d.y, d.z);
          Integral I;
          integrate(cb, dcdt, t_min, t_max, I);
          const float lo = fwd ? 0.f : kMinVal;
          out = make_float4(clipf(I.cer * I.w0 + I.csr * I.w1, lo, kMaxVal),
                            clipf(I.ceg * I.w0 + I.csg * I.w1, lo, kMaxVal),
                            clipf(I.ceb * I.w0 + I.csb * I.w1, lo, kMaxVal), I.od);
          out_t = make_float2(t_min, t_max);
          out_p = pack_item(fmin, fmax, k, p);
        }
        if (MODE == kModeError && hit) out.x = out.y = out.z = 0.0f;  // (weight, counted) filled by phase 1
        s.item[i] = out;
        if (AUX || !fwd || MODE == kModeError) {
          s.itemt[i] = out_t;
          s.itemp[i] = out_p;
        }
      }
    };

    float Cr = 0.f, Cg = 0.f, Cb = 0.f, logT = 0.f;
    float nd0 = 0.f, nd1 = 0.f, nd2 = 0.f, nd3 = 0.f, en0 = 0.f, en1 = 0.f, en2 = 0.f, en3 = 0.f;

    // =============== forward (front to back) ===============
    if (MODE == kModeForward || MODE == kModeTrain) {
      bool alive = valid;
      // custom aux channels accumulate in place in the output row of the pixel
      // (rasterize_compute.wgsl:458-462), so they start at zero
      float* aux_px = nullptr;
      if (AUX && a.aux && a.aux_dim > 0 && valid) {
        aux_px = a.aux + pix * (size_t)(8 + a.aux_dim) + 8;
        for (int ai = 0; ai < a.aux_dim; ++ai) aux_px[ai] = 0.0f;
      }
      if (re > rs) {
        {
          const int nb0 = (int)min((uint32_t)kBatch, re - rs);
          issue(0, nb0, load_idx(re - 1u, nb0, -1), a.spans_fwd + (size_t)(re - (uint32_t)nb0) * kSpanRec);
        }
        uint32_t idx_next = 0u;  // record indices of the batch after the current one
        if (re - rs > (uint32_t)kBatch) {
          const uint32_t h1 = re - (uint32_t)kBatch;
          idx_next = load_idx(h1 - 1u, (int)min((uint32_t)kBatch, h1 - rs), -1);
        }
        int b = 0;
        for (uint32_t hi = re; hi > rs;) {
          const int buf = b & 1;
          const int nb = (int)min((uint32_t)kBatch, hi - rs);
          const uint32_t next_hi = hi - (uint32_t)nb;
          wait_buf(buf);
          if (failed) break;
          load_spans(buf, nb, true);
          prefixes(nb, true);
          __syncthreads();
          // the next batch's copies, after span_pf has been read
          if (next_hi > rs) {
            const int nbn = (int)min((uint32_t)kBatch, next_hi - rs);
            issue(buf ^ 1, nbn, idx_next, a.spans_fwd + (size_t)(next_hi - (uint32_t)nbn) * kSpanRec);
            const uint32_t h2 = next_hi - (uint32_t)nbn;
            if (h2 > rs) idx_next = load_idx(h2 - 1u, (int)min((uint32_t)kBatch, h2 - rs), -1);
          }
          int k1 = sub_end(0, nb);
          fill(0, k1);
          __syncthreads();
          for (int k0 = 0; k0 < nb;) {
            phase0(buf, k0, k1, true);
            __syncthreads();
            // phase 1: composite this pixel's items nearest first
            if (alive) {
              const uint32_t base = s.toff[k0];
              uint32_t m = s.pmask[pl] & ((k1 >= 32 ? 0xffffffffu : ((1u << k1) - 1u)) & ~((1u << k0) - 1u));
              while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1u;
                if (logT < -13.8f) { alive = false; break; }
                const uint32_t it = item_of(k, base);
                const float4 c = s.item[it];
                if (c.w < 0.0f) continue;  // ray miss
                const float Tj = __expf(fmaxf(logT, -88.0f));
                if (Tj >= 1e-6f) {
                  Cr += c.x * Tj; Cg += c.y * Tj; Cb += c.z * Tj;
                  logT -= c.w;
                  if (AUX) {
                    const float2 c2 = s.itemt[it];
                    const float t_min = c2.x, t_max = c2.y;
                    const int entry = (int)(s.itemp[it] & 7u);
                    const float od = c.w;
                    const float alpha_t = __expf(-od);  // as the intersection phase computed it
                    const float ph = fabsf(od) < 0.02f
                                         ? 1.0f + od * (-0.5f + od * (1.0f / 6.0f + od * (-1.0f / 24.0f)))
                                         : clipf(__fdividef(1.0f - alpha_t, od), kMinVal, kMaxVal);
                    const float w0 = ph - alpha_t, w1 = 1.0f - ph;
                    const float alpha = 1.0f - alpha_t;
                    float enx = 0.f, eny = 0.f, enz = 0.f;
                    if (entry < 4) {
                      const float4 n = s.view[buf][k].nrm[entry];
                      const float l = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
                      enx = -n.x / l; eny = -n.y / l; enz = -n.z / l;
                    }
                    const float ta = Tj * alpha;
                    nd0 += ta * enx; nd1 += ta * eny; nd2 += ta * enz;
                    nd3 += Tj * (w0 * t_max + w1 * t_min);
                    const float wt = alpha * Tj;
                    const float cmid = (t_min + t_max) * 0.5f;
                    const float wc = wt * cmid;
                    en0 += wt;
                    en1 += wt > 1e-20f ? wt * logf(wt) : 0.0f;
                    en2 += wt * cmid;
                    en3 += wc > 1e-20f ? wc * logf(wc) : 0.0f;
                    if (aux_px) {
                      const float* ad = a.aux_data + (size_t)s.view[buf][k].meta.x * a.aux_dim;
                      for (int ai = 0; ai < a.aux_dim; ++ai) aux_px[ai] += ta * ad[ai];
                    }
                  }
                }
              }
            }
            const int k2 = k1 < nb ? sub_end(k1, nb) : nb;
            if (k1 < nb) fill(k1, k2);
            __syncthreads();
            k0 = k1;
            k1 = k2;
          }
          hi = next_hi;
          ++b;
          // all pixels saturated: the remaining tets would all be skipped
          if (__syncthreads_count(alive && logT >= -13.8f) == 0) {
            if (hi > rs) wait_buf(buf ^ 1);  // drain the prefetch already in flight
            break;
          }
        }
      }
      if (valid && (MODE == kModeForward || a.rgba != nullptr)) {
        const float A = 1.0f - safe_exp(logT);
        reinterpret_cast<float4*>(a.rgba)[pix] = make_float4(Cr, Cg, Cb, A);
        if (AUX && a.aux && a.aux_dim == 0) {
          reinterpret_cast<float4*>(a.aux)[2 * pix] = make_float4(nd0, nd1, nd2, nd3);
          reinterpret_cast<float4*>(a.aux)[2 * pix + 1] = make_float4(en0, en1, en2, en3);
        } else if (AUX && a.aux) {  // [normal.xyz, depth, entropy.4, custom...] (:486-500)
          float* o = a.aux + pix * (size_t)(8 + a.aux_dim);
          o[0] = nd0; o[1] = nd1; o[2] = nd2; o[3] = nd3;
          o[4] = en0; o[5] = en1; o[6] = en2; o[7] = en3;
        }
      }
    }

    // =============== error statistics (front to back) ===============
    // crates/rmesh-error/src/wgsl/error_tiled_compute.wgsl:90-373: the forward's
    // walk with a -5.5 log-transmittance cut; each covered pixel with T >= 1e-6
    // gives its tet the weight w = T * od.  Phase 1 (per pixel, in order) sets
    // the item to (w, 1); phase 2 reduces per tet (w, w pe, w pe^2, w se,
    // w entry, w exit, count, max 65535 w) and the flush adds them to tet_err /
    // tet_count.
    if (MODE == kModeError) {
      bool alive = valid;
      if (in_tile) s.pdl[pl] = valid ? make_float2(a.pixel_err[pix], a.ssim_err[pix]) : make_float2(0.f, 0.f);
      if (re > rs) {
        {
          const int nb0 = (int)min((uint32_t)kBatch, re - rs);
          issue(0, nb0, load_idx(re - 1u, nb0, -1), a.spans_fwd + (size_t)(re - (uint32_t)nb0) * kSpanRec);
        }
        uint32_t idx_next = 0u;
        if (re - rs > (uint32_t)kBatch) {
          const uint32_t h1 = re - (uint32_t)kBatch;
          idx_next = load_idx(h1 - 1u, (int)min((uint32_t)kBatch, h1 - rs), -1);
        }
        int b = 0;
        for (uint32_t hi = re; hi > rs;) {
          const int buf = b & 1;
          const int nb = (int)min((uint32_t)kBatch, hi - rs);
          const uint32_t next_hi = hi - (uint32_t)nb;
          wait_buf(buf);
          if (failed) break;
          load_spans(buf, nb, true);
          prefixes(nb, true);
          __syncthreads();
          if (next_hi > rs) {
            const int nbn = (int)min((uint32_t)kBatch, next_hi - rs);
            issue(buf ^ 1, nbn, idx_next, a.spans_fwd + (size_t)(next_hi - (uint32_t)nbn) * kSpanRec);
            const uint32_t h2 = next_hi - (uint32_t)nbn;
            if (h2 > rs) idx_next = load_idx(h2 - 1u, (int)min((uint32_t)kBatch, h2 - rs), -1);
          }
          int k1 = sub_end(0, nb);
          fill(0, k1);
          __syncthreads();
          for (int k0 = 0; k0 < nb;) {
            const uint32_t base = s.toff[k0];
            const uint32_t n_items = s.toff[k1] - base;
            phase0(buf, k0, k1, true);
            __syncthreads();
            if (alive) {
              uint32_t m = s.pmask[pl] & ((k1 >= 32 ? 0xffffffffu : ((1u << k1) - 1u)) & ~((1u << k0) - 1u));
              while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1u;
                if (logT < -5.5f) break;
                const uint32_t it = item_of(k, base);
                const float od = s.item[it].w;
                if (od < 0.0f) continue;  // ray miss
                const float Tj = __expf(clipf(logT, -88.0f, kLogMax));
                if (Tj >= 1e-6f) {
                  s.item[it] = make_float4(Tj * od, 1.0f, 0.0f, od);
                  logT -= od;
                }
              }
              if (logT < -5.5f) alive = false;
            }
            __syncthreads();
            // phase 2: per-tet sums of the item statistics (12 columns; column 11
            // is a maximum), a segment of rows per lane as in the adjoint
            float(*red)[kRedCols] = s.red[warp];
            for (uint32_t chunk = (uint32_t)warp * 32u; chunk < n_items; chunk += (uint32_t)NT) {
              const uint32_t i = chunk + (uint32_t)lane;
              float m[kMomHalf];
#pragma unroll
              for (int q = 0; q < kMomHalf; ++q) m[q] = 0.0f;
              int k = -1;
              if (i < n_items) {
                const float4 st = s.item[i];
                const float2 ix = s.itemt[i];
                const uint32_t pk = s.itemp[i];
                k = (int)((pk >> 5) & 31u);
                if (st.y > 0.5f) {
                  const int p = (int)(pk >> 10);
                  const float w = st.x;
                  const float4 d = s.pdir[p];
                  const float2 e = s.pdl[p];
                  const float ox = camx + d.x * V.min_t, oy = camy + d.y * V.min_t, oz = camz + d.z * V.min_t;
                  m[0] = w;
                  m[1] = w * e.x;
                  m[2] = w * e.x * e.x;
                  m[3] = w * e.y;
                  m[4] = w * (ox + d.x * ix.x); m[5] = w * (oy + d.y * ix.x); m[6] = w * (oz + d.z * ix.x);
                  m[7] = w * (ox + d.x * ix.y); m[8] = w * (oy + d.y * ix.y); m[9] = w * (oz + d.z * ix.y);
                  m[10] = 1.0f;
                  m[11] = __int_as_float(__float2int_rz(65535.0f * w));
                }
              }
              const int kp = __shfl_up_sync(0xffffffffu, k, 1);
              const unsigned heads = __ballot_sync(0xffffffffu, k >= 0 && (lane == 0 || kp != k));
              const int n_rows = __popc(__ballot_sync(0xffffffffu, k >= 0));
#pragma unroll
              for (int q = 0; q < kMomHalf; ++q) red[lane][q] = m[q];
              red[lane][kMomHalf] = __int_as_float(k);
              __syncwarp();
              const int wq = lane & 15, wr0 = (lane >> 4) * 16;
              const int wr1 = min(wr0 + 16, n_rows);
              if (wq < kMomHalf && wr0 < wr1) {
                for (int r0 = wr0; r0 < wr1;) {
                  const unsigned later = heads & ~((2u << r0) - 1u);
                  const int r1 = later ? min(__ffs(later) - 1, wr1) : wr1;
                  const int kk = __float_as_int(red[r0][kMomHalf]);
                  if (wq == 11) {
                    int mx = 0;
                    for (int row = r0; row < r1; ++row) mx = max(mx, __float_as_int(red[row][wq]));
                    if (mx > 0) atomicMax(reinterpret_cast<int*>(&s.mom[kk][11]), mx);
                  } else {
                    float sum = 0.0f;
                    for (int row = r0; row < r1; ++row) sum += red[row][wq];
                    if (sum != 0.0f) atomicAdd(&s.mom[kk][wq], sum);
                  }
                  r0 = r1;
                }
              }
              __syncwarp();
            }
            const int k2 = k1 < nb ? sub_end(k1, nb) : nb;
            if (k1 < nb) fill(k1, k2);
            __syncthreads();
            k0 = k1;
            k1 = k2;
          }
          // flush the batch's per-tet sums
          if (tid < nb) {
            float* mm = s.mom[tid];
            if (mm[10] != 0.0f) {
              const TetView& tv = s.view[buf][tid];
              const uint32_t t = tv.meta.x;
              const TetRec r = a.rec[t];
              const float cx = (r.a.x + r.b.x + r.c.x + r.d.x) * 0.25f, cy = (r.a.y + r.b.y + r.c.y + r.d.y) * 0.25f,
                          cz = (r.a.z + r.b.z + r.c.z + r.d.z) * 0.25f;
              float* e = a.tet_err + 16 * (size_t)t;
              atomicAdd(e + 0, mm[0]); atomicAdd(e + 1, mm[1]); atomicAdd(e + 2, mm[2]); atomicAdd(e + 5, mm[3]);
              atomicAdd(e + 6, mm[4]); atomicAdd(e + 7, mm[5]); atomicAdd(e + 8, mm[6]);
              atomicAdd(e + 9, mm[7]); atomicAdd(e + 10, mm[8]); atomicAdd(e + 11, mm[9]);
              atomicAdd(e + 12, mm[0]);
              atomicAdd(e + 13, mm[0] * cx); atomicAdd(e + 14, mm[0] * cy); atomicAdd(e + 15, mm[0] * cz);
              atomicAdd(a.tet_count + 2 * (size_t)t, (int)mm[10]);
              atomicMax(a.tet_count + 2 * (size_t)t + 1, __float_as_int(mm[11]));
            }
#pragma unroll
            for (int q = 0; q < kMomHalf; ++q) mm[q] = 0.0f;
          }
          hi = next_hi;
          ++b;
          if (__syncthreads_count(alive) == 0) {  // every pixel below the cut
            if (hi > rs) wait_buf(buf ^ 1);
            break;
          }
        }
      }
    }

    // =============== adjoint (back to front) ===============
    if (MODE == kModeBackward || MODE == kModeTrain) {
      float dlr = 0.f, dlg = 0.f, dlb = 0.f, dlogT = 0.f;
      if (MODE == kModeTrain) {
        float lsum = 0.f;
        if (valid) {
          const float A = 1.0f - safe_exp(logT);
          const float gr = a.gt_rgb[3 * pix], gg = a.gt_rgb[3 * pix + 1], gb = a.gt_rgb[3 * pix + 2];
          const float er = Cr - gr, eg = Cg - gg, eb = Cb - gb;
          if (a.hp->loss_type == 0) {
            dlr = (er > 0.f ? 1.f : (er < 0.f ? -1.f : 0.f)) / V.n_pixels;
            dlg = (eg > 0.f ? 1.f : (eg < 0.f ? -1.f : 0.f)) / V.n_pixels;
            dlb = (eb > 0.f ? 1.f : (eb < 0.f ? -1.f : 0.f)) / V.n_pixels;
            lsum = fabsf(er) + fabsf(eg) + fabsf(eb);
          } else {
            dlr = 2.0f * er / V.n_pixels;
            dlg = 2.0f * eg / V.n_pixels;
            dlb = 2.0f * eb / V.n_pixels;
            lsum = er * er + eg * eg + eb * eb;
          }
          logT = logf(fmaxf(1.0f - A, 1e-20f));
          dlogT = -0.0f * (1.0f - A);  // the loss has no alpha term (loss_compute.wgsl:71)
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) s.lsum[warp] = lsum;
        __syncthreads();
        if (tid == 0) {
          double tot = 0.0;
          for (int w = 0; w < NW; ++w) tot += (double)s.lsum[w];
          atomicAdd(&a.counters->loss[view], tot);
        }
      } else if (valid) {
        const float4 img = reinterpret_cast<const float4*>(a.rgba)[pix];
        const float4 dl = reinterpret_cast<const float4*>(a.dl_rgba)[pix];
        Cr = img.x; Cg = img.y; Cb = img.z;
        logT = logf(fmaxf(1.0f - img.w, 1e-20f));
        dlogT = -dl.w * (1.0f - img.w);
        dlr = dl.x; dlg = dl.y; dlb = dl.z;
      }
      if (in_tile) {
        s.pdir[pl].w = dlr;
        s.pdl[pl] = make_float2(dlg, dlb);
      }
      if (re > rs) {
        __syncthreads();  // the forward's last reads of the copy buffers
        {
          const int nb0 = (int)min((uint32_t)kBatch, re - rs);
          issue(0, nb0, load_idx(rs, nb0, +1), a.spans_adj + (size_t)rs * kSpanRec);
        }
        uint32_t idx_next = 0u;
        if (re - rs > (uint32_t)kBatch) {
          const uint32_t l1 = rs + (uint32_t)kBatch;
          idx_next = load_idx(l1, (int)min((uint32_t)kBatch, re - l1), +1);
        }
        int b = 0;
        for (uint32_t lo = rs; lo < re;) {
          const int buf = b & 1;
          const int nb = (int)min((uint32_t)kBatch, re - lo);
          const uint32_t next_lo = lo + (uint32_t)nb;
          wait_buf(buf);
          if (failed) break;
          // the flush reads this batch's tet records (vertex positions): start
          // bringing them into L1 now, one thread per tet
          if (tid < nb) {
            const TetRec* rp = a.rec + s.view[buf][tid].meta.x;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(rp));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(reinterpret_cast<const char*>(rp) + 32));
          }
          // adjoint: edge crossings only (backward_tiled_compute.wgsl:241-299)
          load_spans(buf, nb, false);
          prefixes(nb, false);
          __syncthreads();
          // the next batch's copies, after span_pf has been read
          if (next_lo < re) {
            const int nbn = (int)min((uint32_t)kBatch, re - next_lo);
            issue(buf ^ 1, nbn, idx_next, a.spans_adj + (size_t)next_lo * kSpanRec);
            const uint32_t l2 = next_lo + (uint32_t)nbn;
            if (l2 < re) idx_next = load_idx(l2, (int)min((uint32_t)kBatch, re - l2), +1);
          }
          int k1 = sub_end(0, nb);
          fill(0, k1);
          __syncthreads();
          for (int k0 = 0; k0 < nb;) {
            const uint32_t base = s.toff[k0];
            const uint32_t n_items = s.toff[k1] - base;
            phase0(buf, k0, k1, false);
            __syncthreads();
            // phase 1: undo this pixel's items farthest first
            if (valid) {
              uint32_t m = s.pmask[pl] & ((k1 >= 32 ? 0xffffffffu : ((1u << k1) - 1u)) & ~((1u << k0) - 1u));
              while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1u;
                const uint32_t it = item_of(k, base);
                const float4 c = s.item[it];
                if (c.w < 0.0f) continue;  // ray miss: no state change, no gradient
                const float prev_logT = fminf(logT + c.w, 0.0f);
                const float t_prev = __expf(fmaxf(prev_logT, -88.0f));
                Cr -= c.x * t_prev; Cg -= c.y * t_prev; Cb -= c.z * t_prev;
                logT = prev_logT;
                if (t_prev >= 1e-6f) {
                  const float d_od_state = -dlogT;
                  // custom aux channels (aux += T alpha a[tet], rasterize_compute.wgsl:458-462)
                  // continue the transmittance chain like a colour alpha a[tet]:
                  // aux_s = sum_ai dl_aux[pixel][ai] a[tet][ai]
                  float aux_s = 0.0f, aux_w = 0.0f;
                  if (AUX && MODE == kModeBackward && a.dl_aux) {
                    const float* dla = a.dl_aux + pix * (size_t)a.aux_dim;
                    const float* ad = a.aux_data + (size_t)s.view[buf][k].meta.x * a.aux_dim;
                    for (int ai = 0; ai < a.aux_dim; ++ai) aux_s += dla[ai] * ad[ai];
                    aux_w = (1.0f - __expf(-c.w)) * aux_s;  // alpha * aux_s
                  }
                  dlogT = clipf(dlogT + (dlr * c.x + dlg * c.y + dlb * c.z + aux_w) * t_prev, kMinVal, kMaxVal);
                  s.item[it] = make_float4(t_prev, d_od_state, 1.0f, aux_s);
                } else {
                  s.item[it] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);  // no gradient
                }
              }
            }
            __syncthreads();
            // phase 2: per-item adjoint, item-parallel in 32-item warp chunks.
            // Vertex gradients enter through moments: for a face (a, b, c) with
            // unflipped normal n, hit h = cam + d t and s = dT / (n.d), the item
            // adds s (a-h) x (c-a) to vertex b, s (a-h) x (a-b) to c and
            // s ((a-h) x (b-c) + n) to a (backward_tiled_compute.wgsl:506-533).
            // Since a - h = (a - cam) - t d, the sum over a tet's items needs only
            // S = sum s and P = sum s t d per face; the vertex gradients are
            // rebuilt from them once per tet at flush time.  Moments per item:
            //  [0] density  [1..3] base colour  [4] sum(sb)  [5..7] d * d(dc/dt)
            //  [8 + 4f] S_f  [9 + 4f .. 11 + 4f] P_f   (f = face 0..3)
            // Each tet's items are cut into runs of at most R consecutive items
            // (its pixels along its rows), R chosen so that the sub-batch has at
            // most one run per thread; thread t takes run t and sums its items'
            // moments: the 8 tet moments in registers, the (S, P) of the 4 faces
            // in the lane's row of the warp buffer (an item adds to the rows of
            // its entry and exit faces by address, where registers would need a
            // select over all 16 sums per side).  The runs' sums (lanes in run
            // order, so a tet's lanes are adjacent) are then combined per warp
            // through that buffer, half of the moments at a time: lane (h, q)
            // with q < kMomHalf walks one column over rows [16h, 16h + 16) and adds
            // a partial sum to the tet's moment at every tet boundary and at the
            // end of its rows.
            {
              const int nsub = k1 - k0;
              const uint32_t R = max(1u, (n_items + (uint32_t)(NT - nsub) - 1u) / (uint32_t)(NT - nsub));
              float(*red)[kRedCols] = s.red[warp];
              // cumulative run counts of the sub-batch's tets (each warp its own copy)
              int* crun = reinterpret_cast<int*>(&red[0][0]);
              {
                int cnt = 0;
                if (lane < nsub) cnt = (int)((s.toff[k0 + lane + 1] - s.toff[k0 + lane] + R - 1u) / R);
                int x = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                  const int y = __shfl_up_sync(0xffffffffu, x, o);
                  if (lane >= o) x += y;
                }
                crun[lane + 1] = x;
                if (lane == 0) crun[0] = 0;
                __syncwarp();
              }
              int k = -1;
              uint32_t i0 = 0, i1 = 0;
              if (tid < crun[nsub]) {
                int lo = 0, hi = nsub;  // crun[lo] <= tid < crun[hi]
                while (hi - lo > 1) {
                  const int mid = (lo + hi) >> 1;
                  if (crun[mid] <= tid) lo = mid; else hi = mid;
                }
                k = k0 + lo;
                i0 = s.toff[k] - base + (uint32_t)(tid - crun[lo]) * R;
                i1 = min(i0 + R, s.toff[k + 1] - base);
              }
              __syncwarp();  // crun is overwritten by the face sums below
              float acc[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) acc[q] = 0.0f;
              // this lane's face sums live in its row of the warp buffer, so the
              // item's entry / exit face is an address, not a 16-way select
              float* fac = red[lane];
#pragma unroll
              for (int q = 0; q < 16; ++q) fac[q] = 0.0f;
              for (uint32_t i = i0; i < i1; ++i) {
                const float4 st = s.item[i];
                // (t_prev, d_od_state, 1, aux_s) for an item with a gradient; ray misses
                // and items below the transmittance cut have z = 0
                if (!(st.z > 0.5f)) continue;
                const float2 ix = s.itemt[i];
                const uint32_t pk = s.itemp[i];
                const int p = (int)(pk >> 10);
                int fmin = (int)(pk & 7u);
                const int fmax = (int)((pk >> 3) & 3u);
                if (fmin == 4) fmin = 0;  // reference keeps min_face = 0 when no face enters
                const float t_min = ix.x, t_max = ix.y;
                const float t_prev = st.x, d_od_state = st.y;
                const float4 d = s.pdir[p];
                const float2 dgb = s.pdl[p];
                const TetView& tv = s.view[buf][k];
                const float4 cb = tv.cb;
                const float4 gg = tv.gm;
                const float dcdt = dot3x(gg.x, gg.y, gg.z, d.x, d.y, d.z);
                Integral I;
                integrate(cb, dcdt, t_min, t_max, I);
                const float dcpr = clipf(d.w * t_prev, kMinVal, kMaxVal);
                const float dcpg = clipf(dgb.x * t_prev, kMinVal, kMaxVal);
                const float dcpb = clipf(dgb.y * t_prev, kMinVal, kMaxVal);
                float dph;
                if (fabsf(I.od) < 0.02f)
                  dph = -0.5f + I.od * (1.0f / 3.0f + I.od * (-1.0f / 8.0f + I.od * (1.0f / 30.0f)));
                else
                  dph = clipf(__fdividef(I.alpha_t * (I.od + 1.0f) - 1.0f, I.od * I.od), kMinVal, kMaxVal);
                const float dw0 = dph + I.alpha_t, dw1 = -dph;
                const float d_od_int = dcpr * (I.cer * dw0 + I.csr * dw1) + dcpg * (I.ceg * dw0 + I.csg * dw1) +
                                       dcpb * (I.ceb * dw0 + I.csb * dw1);
                float d_od_aux = 0.0f;
                if (AUX && MODE == kModeBackward && a.dl_aux) {
                  // the aux channels' own terms: d od += T_prev alpha_t aux_s (d alpha / d od =
                  // alpha_t); d a[tet][ai] += dl_aux[pixel][ai] T_prev alpha
                  d_od_aux = t_prev * I.alpha_t * st.w;
                  const int pr = p / TS, pc = p - (p / TS) * TS;
                  const size_t gp = (size_t)V.pix_base + (size_t)(tile_y * (uint32_t)TS + (uint32_t)pr) * (size_t)V.W +
                                    (size_t)(tile_x * (uint32_t)TS + (uint32_t)pc);
                  const float* dla = a.dl_aux + gp * (size_t)a.aux_dim;
                  float* dst = a.d_aux + (size_t)tv.meta.x * a.aux_dim;
                  const float wa = t_prev * (1.0f - I.alpha_t);
                  for (int ai = 0; ai < a.aux_dim; ++ai) {
                    const float v = dla[ai] * wa;
                    if (v != 0.0f) atomicAdd(dst + ai, v);
                  }
                }
                const float d_od = clipf(d_od_state + d_od_int + d_od_aux, kMinVal, kMaxVal);
                const bool active = (I.od_raw >= 1e-8f) && (I.od_raw <= 88.0f);
                const float d_od_raw = active ? d_od : 0.0f;
                const float d_dist = clipf(d_od_raw * cb.w, kMinVal, kMaxVal);
                float d_tmin = -d_dist, d_tmax = d_dist;
                const float dsr = I.csr_r > 0.f ? dcpr * I.w1 : 0.f, dsg = I.csg_r > 0.f ? dcpg * I.w1 : 0.f,
                            dsb = I.csb_r > 0.f ? dcpb * I.w1 : 0.f;
                const float der = I.cer_r > 0.f ? dcpr * I.w0 : 0.f, deg = I.ceg_r > 0.f ? dcpg * I.w0 : 0.f,
                            deb = I.ceb_r > 0.f ? dcpb * I.w0 : 0.f;
                const float dbr = dsr + der, dbg = dsg + deg, dbb = dsb + deb;
                const float ss = dsr + dsg + dsb, se = der + deg + deb;
                const float d_dcdt = ss * t_min + se * t_max;
                d_tmin += ss * dcdt;
                d_tmax += se * dcdt;
                acc[0] += clipf(d_od_raw * I.dist, kMinVal, kMaxVal);
                acc[1] += clipf(dbr, kMinVal, kMaxVal);
                acc[2] += clipf(dbg, kMinVal, kMaxVal);
                acc[3] += clipf(dbb, kMinVal, kMaxVal);
                acc[4] += dbr + dbg + dbb;
                acc[5] += d.x * d_dcdt;
                acc[6] += d.y * d_dcdt;
                acc[7] += d.z * d_dcdt;
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                  const int f = side == 0 ? fmin : fmax;
                  const float dt = side == 0 ? d_tmin : d_tmax;
                  const float tt = side == 0 ? t_min : t_max;
                  const float4 nf = tv.nrm[f];
                  const float den = (face_flipped(tv, f) ? -1.0f : 1.0f) * (nf.x * d.x + nf.y * d.y + nf.z * d.z);
                  const float inv_den = fabsf(den) < kTiny ? clipf(1.0f / kTiny, kMinVal, kMaxVal)
                                                           : clipf(__fdividef(1.0f, den), kMinVal, kMaxVal);
                  const float sv = dt * inv_den, st_ = sv * tt;
                  float* fp = fac + 4 * f;
                  fp[0] += sv;
                  fp[1] += st_ * d.x;
                  fp[2] += st_ * d.y;
                  fp[3] += st_ * d.z;
                }
              }
              // warp combine of the runs' sums (lanes without a run come last)
              const int kp = __shfl_up_sync(0xffffffffu, k, 1);
              const unsigned heads = __ballot_sync(0xffffffffu, k >= 0 && (lane == 0 || kp != k));
              const int n_rows = __popc(__ballot_sync(0xffffffffu, k >= 0));
              red[lane][16] = __int_as_float(k);
              __syncwarp();
              if (n_rows > 0) {
                const int wq = lane & 15, wr0 = (lane >> 4) * 16;
                const int wr1 = min(wr0 + 16, n_rows);
#pragma unroll
                for (int hm = 0; hm < 2; ++hm) {
                  // pass 0: faces 1..3 (moments 12..23) from columns 4..15; pass 1: the
                  // 8 tet moments, written over columns 4..11, and face 0 (moments
                  // 8..11) from columns 0..3
                  if (hm == 1) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) red[lane][4 + q] = acc[q];
                    __syncwarp();
                  }
                  if (wq < kMomHalf && wr0 < wr1) {
                    const int col = hm == 0 ? kMomHalf + wq : wq;
                    const int src = hm == 0 ? 4 + wq : (wq < 8 ? 4 + wq : wq - 8);
                    for (int r0 = wr0; r0 < wr1;) {  // one tet segment [r0, r1) at a time
                      const unsigned later = heads & ~((2u << r0) - 1u);
                      const int r1 = later ? min(__ffs(later) - 1, wr1) : wr1;
                      float sum = 0.0f;
                      for (int row = r0; row < r1; ++row) sum += red[row][src];
                      if (sum != 0.0f) atomicAdd(&s.mom[__float_as_int(red[r0][16])][col], sum);
                      r0 = r1;
                    }
                  }
                  __syncwarp();
                }
              }
            }
            const int k2 = k1 < nb ? sub_end(k1, nb) : nb;
            if (k1 < nb) fill(k1, k2);
            __syncthreads();
            k0 = k1;
            k1 = k2;
          }
          // flush: rebuild each tet's 19 gradients from its moments, four threads
          // per tet (thread f takes face f's vertex terms, thread 0 also the
          // density / colour terms), summed by shuffles; thread 0 adds them to the
          // global slot with five 16-byte vector atomics
          for (int t0 = 0; t0 < 4 * kBatch; t0 += NT) {  // block-uniform trip count
            const int task = t0 + tid;
            const int k = task >> 2, f = task & 3;
            const bool live = k < nb;
            float* mm = s.mom[live ? k : 0];
            const float S = live ? mm[8 + 4 * f] : 0.f, Px = live ? mm[9 + 4 * f] : 0.f;
            const float Py = live ? mm[10 + 4 * f] : 0.f, Pz = live ? mm[11 + 4 * f] : 0.f;
            const bool face_any = S != 0.0f || Px != 0.0f || Py != 0.0f || Pz != 0.0f;
            bool any = face_any;
            if (live && f == 0) {
#pragma unroll
              for (int q = 0; q < 8; ++q) any = any || (mm[q] != 0.0f);
            }
            const unsigned grp = (__ballot_sync(0xffffffffu, any) >> (lane & ~3)) & 0xFu;
            float dv[12];
#pragma unroll
            for (int q = 0; q < 12; ++q) dv[q] = 0.0f;
            float out[7];
            const TetView& tv = s.view[buf][live ? k : 0];
            if (live && grp) {
              const TetRec r = a.rec[tv.meta.x];
              if (f == 0) {
                const float4 gg = tv.gm;
                out[0] = mm[0];
                out[1] = mm[1]; out[2] = mm[2]; out[3] = mm[3];
                const float sb = mm[4];
                out[4] = clipf((camx - r.a.x) * sb + mm[5], kMinVal, kMaxVal);
                out[5] = clipf((camy - r.a.y) * sb + mm[6], kMinVal, kMaxVal);
                out[6] = clipf((camz - r.a.z) * sb + mm[7], kMinVal, kMaxVal);
                dv[0] = -gg.x * sb; dv[1] = -gg.y * sb; dv[2] = -gg.z * sb;
              }
              if (face_any) {
                const int ia = kFaces[f][0], ib = kFaces[f][1], ic = kFaces[f][2];
                const float4 va = rec_vertex(r, ia), vb = rec_vertex(r, ib), vc = rec_vertex(r, ic);
                const float4 nf = tv.nrm[f];
                const float sg = face_flipped(tv, f) ? -1.0f : 1.0f;
                // w = (a - cam) S - P
                const float wx = (va.x - camx) * S - Px, wy = (va.y - camy) * S - Py, wz = (va.z - camz) * S - Pz;
                float ux = vc.x - va.x, uy = vc.y - va.y, uz = vc.z - va.z;  // c - a
                const float bx = wy * uz - wz * uy, by = wz * ux - wx * uz, bz = wx * uy - wy * ux;
                ux = va.x - vb.x; uy = va.y - vb.y; uz = va.z - vb.z;  // a - b
                const float cx = wy * uz - wz * uy, cy = wz * ux - wx * uz, cz = wx * uy - wy * ux;
                const float ax = sg * nf.x * S - bx - cx, ay = sg * nf.y * S - by - cy, az = sg * nf.z * S - bz - cz;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  if (q == ia) { dv[3 * q] += ax; dv[3 * q + 1] += ay; dv[3 * q + 2] += az; }
                  if (q == ib) { dv[3 * q] += bx; dv[3 * q + 1] += by; dv[3 * q + 2] += bz; }
                  if (q == ic) { dv[3 * q] += cx; dv[3 * q + 1] += cy; dv[3 * q + 2] += cz; }
                }
              }
            }
#pragma unroll
            for (int q = 0; q < 12; ++q) {
              dv[q] += __shfl_xor_sync(0xffffffffu, dv[q], 1);
              dv[q] += __shfl_xor_sync(0xffffffffu, dv[q], 2);
            }
            if (live && grp && f == 0) {
              float4* dst = reinterpret_cast<float4*>(a.grad_slot + (size_t)tv.meta.x * kGradSlot);
              if (a.vis_dcolor) {  // SH colours: this view's colour gradient of the entry
                const float4 dc = make_float4(out[1], out[2], out[3], 0.0f);
                if (dc.x != 0.f || dc.y != 0.f || dc.z != 0.f) atomicAdd(a.vis_dcolor + tv.meta.y, dc);
                out[1] = out[2] = out[3] = 0.0f;
              }
              float o2[20];
#pragma unroll
              for (int q = 0; q < 7; ++q) o2[q] = out[q];
#pragma unroll
              for (int q = 0; q < 12; ++q) o2[7 + q] = clipf(dv[q], kMinVal, kMaxVal);
              o2[19] = 0.0f;
#pragma unroll
              for (int c = 0; c < 5; ++c) {
                const float4 v4 = make_float4(o2[4 * c], o2[4 * c + 1], o2[4 * c + 2], o2[4 * c + 3]);
                if (v4.x != 0.f || v4.y != 0.f || v4.z != 0.f || v4.w != 0.f) atomicAdd(dst + c, v4);
              }
            }
            if (live) {  // each thread clears what it read
              mm[8 + 4 * f] = 0.f; mm[9 + 4 * f] = 0.f; mm[10 + 4 * f] = 0.f; mm[11 + 4 * f] = 0.f;
              if (f == 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) mm[q] = 0.0f;
              }
            }
          }
          __syncthreads();
          lo = next_lo;
          ++b;
        }
      }
    }
    if (!a.persistent) break;
    __syncthreads();
  }
}

// Span records of every sorted (tile, tet) pair, one per rule: kSpanRows
// one-byte row spans (row_spans) over the rows its tet reaches (the row table rule
// of the tile kernel): the tile kernel bulk-copies a batch's rows with its tet
// records instead of deriving them between block barriers.  Other rows, tets
// with a vertex behind the camera and sentinel slots get empty spans (the tile
// kernel reads none of them).  Each warp takes 32 consecutive pairs; lane l
// sets up pair l, and the warp's (pair, row) tasks are spread over its lanes
// through a prefix of the row counts, so lanes stay busy whatever the rows per
// tet.  The rows go to shared memory; the owner lane then adds, per row, the
// pixels of the rows above it (at most 15 x 16 = 240, one byte) and stores
// the pair's two 32-byte records whole.
// Byte r of the result: the covered pixels of span rows 0..r-1 of v (16
// packed spans, one per byte), four rows per 32-bit word at a time: per byte,
// (hi | 0x80) - lo keeps bit 7 exactly when lo <= hi and holds hi - lo below
// it; the word's prefix sum of the widths is one multiply by 0x01010101 (no
// byte carries: at most 15 x 16 = 240 pixels lie above any row).
__device__ __forceinline__ uint4 rows_above(uint4 v) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
  uint32_t c[4];
  uint32_t acc = 0u;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t lo = (w[q] >> 4) & 0x0F0F0F0Fu, hi = w[q] & 0x0F0F0F0Fu;
    const uint32_t d = (hi | 0x80808080u) - lo;
    const uint32_t mask = ((d & 0x80808080u) >> 7) * 0xFFu;
    const uint32_t width = ((d & 0x7F7F7F7Fu) + 0x01010101u) & mask;
    const uint32_t incl = width * 0x01010101u;
    c[q] = incl - width + acc * 0x01010101u;
    acc += incl >> 24;
  }
  return make_uint4(c[0], c[1], c[2], c[3]);
}

struct PairSpanArgs {
  const ViewParams* views;
  int n_views;
  const uint32_t* keys;              // sorted global tile ids
  const uint32_t* vals;              // the pairs' entry indices (per-view tet records)
  const unsigned long long* n_ptr;   // pair count
  unsigned long long cap;
  const TetView* vis_view;
  uint8_t* spans_fwd;
  uint8_t* spans_adj;
};

__global__ void __launch_bounds__(256) pair_spans_kernel(PairSpanArgs a) {
  static_assert(kSpanRows == 16 && kSpanRec == 32, "16 span bytes + 16 row-offset bytes per pair and rule");
  __shared__ __align__(16) uint8_t s_fwd[256][kSpanRows];
  __shared__ __align__(16) uint8_t s_adj[256][kSpanRows];
  const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
  const unsigned long long n = *a.n_ptr < a.cap ? *a.n_ptr : a.cap;
  const uint4 empty = make_uint4(0xF0F0F0F0u, 0xF0F0F0F0u, 0xF0F0F0F0u, 0xF0F0F0F0u);
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < n;
       base += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long p = base + threadIdx.x;
    *reinterpret_cast<uint4*>(s_fwd[threadIdx.x]) = empty;
    *reinterpret_cast<uint4*>(s_adj[threadIdx.x]) = empty;
    float vpx[4] = {0.f, 0.f, 0.f, 0.f}, vpy[4] = {0.f, 0.f, 0.f, 0.f};
    int valid_cols = 0, r0 = 0, nrows = 0;
    if (p < n) {
      const uint32_t key = a.keys[p];
      if (key != kSentinel) {
        const ViewParams& V = a.views[view_of_tile(a.views, a.n_views, key)];
        const int TS = V.TS;
        const uint32_t local = key - V.tile_base;
        const uint32_t ty = local / (uint32_t)V.tiles_x, tx = local - ty * (uint32_t)V.tiles_x;
        valid_cols = min(TS, V.W - (int)(tx * (uint32_t)TS));
        const int valid_rows = min(TS, V.H - (int)(ty * (uint32_t)TS));
        const TetView* tv = a.vis_view + a.vals[p];
        if (!((__float_as_uint(__ldg(&tv->gm.w)) >> 4) & 1u)) {
          const float4 gx4 = __ldg(&tv->px), gy4 = __ldg(&tv->py);
          const float tile_ox = (float)(tx * (uint32_t)TS), tile_oy = (float)(ty * (uint32_t)TS);
          vpx[0] = gx4.x - tile_ox; vpx[1] = gx4.y - tile_ox; vpx[2] = gx4.z - tile_ox; vpx[3] = gx4.w - tile_ox;
          vpy[0] = gy4.x - tile_oy; vpy[1] = gy4.y - tile_oy; vpy[2] = gy4.z - tile_oy; vpy[3] = gy4.w - tile_oy;
          // the vertices sorted by y (five compare-exchanges), as row_spans takes them
          auto cx = [&](int i, int j) {
            if (vpy[j] < vpy[i]) {
              const float ty = vpy[i], tx = vpx[i];
              vpy[i] = vpy[j]; vpx[i] = vpx[j];
              vpy[j] = ty; vpx[j] = tx;
            }
          };
          cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
          // rows r with floor(ylo) <= r <= floor(yhi), clipped to the image: the
          // only rows the forward's reach rule can accept
          const float ylo = vpy[0], yhi = vpy[3];
          const float flo = fmaxf(floorf(ylo), 0.0f);
          const float fhi = fminf(floorf(yhi), (float)(valid_rows - 1));
          if (flo <= fhi) {
            r0 = (int)flo;
            nrows = (int)fhi - r0 + 1;
          }
        }
      }
    }
    int pre = nrows;  // inclusive prefix of the row counts over the warp's lanes
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, pre, o);
      if (lane >= o) pre += y;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    const int first_row = r0 - (pre - nrows);  // row of task t of this lane's pair: first_row + t
    __syncwarp();  // the records' empty rows are set before any task writes one
    for (int t0 = 0; t0 < total; t0 += 32) {  // warp-uniform trip count
      const int t = t0 + lane;
      int k = 0;  // the lane whose pair owns task t: first inclusive prefix > t
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const int pv = __shfl_sync(0xffffffffu, pre, k + st - 1);
        if (pv <= t) k += st;
      }
      const int row = __shfl_sync(0xffffffffu, first_row, k) + t;
      const int vc = __shfl_sync(0xffffffffu, valid_cols, k);
      float qx[4], qy[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        qx[q] = __shfl_sync(0xffffffffu, vpx[q], k);
        qy[q] = __shfl_sync(0xffffffffu, vpy[q], k);
      }
      if (t < total) row_spans(qx, qy, row, vc, s_fwd[wbase + k][row], s_adj[wbase + k][row]);
    }
    __syncwarp();
    if (p < n) {
      const uint4 vf = *reinterpret_cast<const uint4*>(s_fwd[threadIdx.x]);
      const uint4 va = *reinterpret_cast<const uint4*>(s_adj[threadIdx.x]);
      uint4* df = reinterpret_cast<uint4*>(a.spans_fwd + p * kSpanRec);
      uint4* da = reinterpret_cast<uint4*>(a.spans_adj + p * kSpanRec);
      df[0] = vf;
      df[1] = rows_above(vf);
      da[0] = va;
      da[1] = rows_above(va);
    }
    __syncwarp();  // the stores' reads before the next chunk's rows are reset
  }
}

}  // namespace rm
