// Tiled compositing: forward, adjoint, and the fused forward+loss+adjoint.
//
// Reference kernels restated:
//   forward   crates/rmesh-render/src/wgsl/rasterize_compute.wgsl:92-511
//   loss      crates/rmesh-train/src/wgsl/loss_compute.wgsl:24-72
//   adjoint   crates/rmesh-backward/src/wgsl/backward_tiled_compute.wgsl:154-587
//
// B200 layout: one CTA per tile with ONE THREAD PER PIXEL (TS*TS pixels,
// rounded up to whole warps), per-pixel state in registers instead of shared
// memory, and the tile's tets processed in batches of kBatch.  For each batch
// warp 0 stages the 64-byte tet records and 16-byte colours into shared memory
// with TMA bulk copies (double buffered: batch b+1 is in flight while batch b
// is composited), one thread per tet derives the per-tet quantities (tile-local
// projection, inward face planes, colour base), kBatch*TS threads derive the
// per-row pixel spans exactly as the reference scanline does, and every pixel
// thread then walks the batch.  Barriers: 3 per batch instead of 3 per tet.
//
// Coverage semantics kept from the reference: the forward includes vertices
// inside a pixel row (rasterize_compute.wgsl:236-242) and skips pixels whose
// log-transmittance fell below -13.8 (:257-262, :338); the adjoint uses edge
// crossings only (backward_tiled_compute.wgsl:241-299), takes the ray origin at
// the camera, undoes every covered tet (clamping log T at 0) and skips the
// gradient when the restored transmittance is below 1e-6 (:424-437).
//
// Adjoint reduction: per tet, each warp sums its lanes' 19 partials with a
// butterfly reduce-scatter (31 shuffles, lane l ends with partial l), adds them
// into a shared-memory slot, and after the batch the CTA flushes each tet's
// 20-float slot to global memory with five 16-byte vector atomics.
#pragma once
#include "common.cuh"
#include "project.cuh"
#include "tma.cuh"

namespace rm {

constexpr int kBatch = 32;

enum TileMode : int { kModeForward = 0, kModeBackward = 1, kModeTrain = 2 };

struct TileArgs {
  const ViewParams* views;
  int n_views;
  uint32_t n_tiles;
  const uint2* ranges;
  const uint32_t* pair_val;
  const TetRec* rec;
  const float4* color4;
  uint32_t color_view_stride;  // 0: colours shared by all views; M: per-view colours
  float* rgba;                 // [pixels][4] (forward output; optional in train mode)
  float* aux;                  // [pixels][8] (optional, forward only)
  const float* dl_rgba;        // [pixels][4] (backward mode)
  const float* gt_rgb;         // [pixels][3] (train mode)
  float* grad_slot;            // [M][kGradSlot]
  float* dcolor_slot;          // optional [views*M][4] per-view colour gradient (SH mode)
  Counters* counters;
  const AdamParams* hp;
  int persistent;
};

template <int TS>
struct __align__(16) TileSmem {
  TetRec rec[2][kBatch];
  float4 col[2][kBatch];
  float4 nrm[kBatch][4];  // inward face normal xyz, num = dot(n, va - cam)
  float4 cb[kBatch];      // colour + dot(g, cam - v0), density
  float4 gr[kBatch];      // g xyz, flip bits (as uint) in w
  float px[kBatch][4];
  float py[kBatch][4];
  float4 acc[kBatch][5];  // adjoint partial sums (20 floats per tet)
  uint32_t tet[2][kBatch];
  uint32_t behind[kBatch];
  short2 span[kBatch][TS];
  uint64_t bar[2];
  float red[16];
  uint32_t tile;
  uint32_t flags;
};

// Butterfly reduce-scatter over 32 lanes: on return lane l holds the warp sum of v[l]
// (v[l] for l >= N is taken as zero).
template <int N>
__device__ __forceinline__ float warp_reduce_scatter(const float (&v)[N], int lane) {
  float a[16];
  const bool b4 = (lane >> 4) & 1;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const float lo = i < N ? v[i] : 0.0f;
    const float hi = (i + 16) < N ? v[i + 16] : 0.0f;
    const float send = b4 ? lo : hi;
    const float keep = b4 ? hi : lo;
    a[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float b[8];
  const bool b3 = (lane >> 3) & 1;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float send = b3 ? a[i] : a[i + 8];
    const float keep = b3 ? a[i + 8] : a[i];
    b[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float c[4];
  const bool b2 = (lane >> 2) & 1;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float send = b2 ? b[i] : b[i + 4];
    const float keep = b2 ? b[i + 4] : b[i];
    c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  float d[2];
  const bool b1 = (lane >> 1) & 1;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float send = b1 ? c[i] : c[i + 2];
    const float keep = b1 ? c[i + 2] : c[i];
    d[i] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  const bool b0 = lane & 1;
  const float send = b0 ? d[0] : d[1];
  const float keep = b0 ? d[1] : d[0];
  return keep + __shfl_xor_sync(0xffffffffu, send, 1);
}

// dot(n, va - o) for face f of a staged record (ray origin o off the camera).
__device__ __forceinline__ float face_num_offset(const TetRec& r, int f, const float4& n, float ox, float oy,
                                                 float oz) {
  const int ia = kFaces[f][0];
  const float4 v = ia == 0 ? r.a : (ia == 1 ? r.b : (ia == 2 ? r.c : r.d));
  return dot3x(n.x, n.y, n.z, fs(v.x, ox), fs(v.y, oy), fs(v.z, oz));
}

template <int TS, int MODE, bool AUX>
__global__ void __launch_bounds__(((TS * TS + 31) / 32) * 32) tile_kernel(TileArgs a) {
  constexpr int NT = ((TS * TS + 31) / 32) * 32;
  constexpr int NW = NT / 32;
  __shared__ TileSmem<TS> s;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int prow = tid / TS < TS ? tid / TS : TS - 1;  // padding threads read a real row, never use it
  const int pcol = tid - (tid / TS) * TS;

  if (tid == 0) {
    mbar_init(&s.bar[0], 1);
    mbar_init(&s.bar[1], 1);
    fence_mbar_init();
  }
  for (int i = tid; i < kBatch * 5; i += NT) (&s.acc[0][0])[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  uint32_t phase[2] = {0u, 0u};
  bool failed = false;

  uint32_t first_tile = blockIdx.x;
  while (true) {
    if (tid == 0) s.tile = a.persistent ? atomicAdd(&a.counters->tile_ticket, 1u) : first_tile;
    __syncthreads();
    const uint32_t g = s.tile;
    if (g >= a.n_tiles || failed) break;
    const int view = view_of_tile(a.views, a.n_views, g);
    const ViewParams& V = a.views[view];
    const uint32_t local_tile = g - V.tile_base;
    const uint32_t tile_y = local_tile / (uint32_t)V.tiles_x;
    const uint32_t tile_x = local_tile - tile_y * (uint32_t)V.tiles_x;
    const float tile_ox = (float)(tile_x * (uint32_t)TS), tile_oy = (float)(tile_y * (uint32_t)TS);
    const uint32_t px = tile_x * (uint32_t)TS + (uint32_t)pcol;
    const uint32_t py = tile_y * (uint32_t)TS + (uint32_t)prow;
    const bool valid = tid < TS * TS && px < (uint32_t)V.W && py < (uint32_t)V.H;
    const size_t pix = (size_t)V.pix_base + (size_t)py * (size_t)V.W + px;
    const uint2 range = a.ranges[g];
    const uint32_t rs = range.x, re = range.y;

    // pixel ray (rasterize_compute.wgsl:343-349), explicitly rounded: the ray and
    // the plane hits below feed t_max - t_min, which cancels for thin tets, so
    // they are evaluated exactly as the reference's left-to-right float math.
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
    const float camx = V.cam[0], camy = V.cam[1], camz = V.cam[2];
    // forward ray origin cam + dir * min_t (rasterize_compute.wgsl:352); the
    // adjoint keeps the origin at the camera (backward_tiled_compute.wgsl:377)
    const bool has_min_t = V.min_t != 0.0f;
    const float ox = fa(camx, fm(dx, V.min_t)), oy = fa(camy, fm(dy, V.min_t)), oz = fa(camz, fm(dz, V.min_t));

    // ---------------- per-tile batch machinery ----------------
    // dir = -1: front-to-back from re-1 down to rs (forward); +1: rs up to re-1 (adjoint)
    auto issue = [&](int buf, uint32_t first, int nb, int dir) {
      if (warp == 0) {
        if (lane == 0) {
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&s.bar[buf], (uint32_t)nb * (uint32_t)(sizeof(TetRec) + sizeof(float4)));
        }
        __syncwarp();
        if (lane < nb) {
          const uint32_t pos = dir < 0 ? first - (uint32_t)lane : first + (uint32_t)lane;
          const uint32_t t = a.pair_val[pos];
          s.tet[buf][lane] = t;
          bulk_copy_g2s(&s.rec[buf][lane], a.rec + t, (uint32_t)sizeof(TetRec), &s.bar[buf]);
          bulk_copy_g2s(&s.col[buf][lane], a.color4 + (size_t)a.color_view_stride * view + t,
                        (uint32_t)sizeof(float4), &s.bar[buf]);
        }
      }
    };
    // every thread waits on the phase; the outcome is made block-uniform
    auto wait_buf = [&](int buf) {
      const bool ok = mbar_wait_bounded(&s.bar[buf], phase[buf], 1u << 20);
      phase[buf] ^= 1u;
      if (__syncthreads_or(!ok)) {
        failed = true;
        if (tid == 0) atomicOr(&a.counters->err, kErrSpinTimeout);
      }
    };
    // per-tet setup (thread k < nb) from staged record
    auto setup = [&](int buf, int nb) {
      if (tid < nb) {
        const int k = tid;
        const TetRec r = s.rec[buf][k];
        const float4 col = s.col[buf][k];
        const float vx[4] = {r.a.x, r.b.x, r.c.x, r.d.x};
        const float vy[4] = {r.a.y, r.b.y, r.c.y, r.d.y};
        const float vz[4] = {r.a.z, r.b.z, r.c.z, r.d.z};
        float cl[4][4];
        bool behind = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          clip_exact(V.vp, vx[q], vy[q], vz[q], cl[q]);
          behind = behind || (cl[q][3] <= 0.0f);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float ppx = 0.f, ppy = 0.f;
          if (!behind) {
            ppx = fs(fm(fm(fa(fdv(cl[q][0], cl[q][3]), 1.0f), 0.5f), V.Wf), tile_ox);
            ppy = fs(fm(fm(fs(1.0f, fdv(cl[q][1], cl[q][3])), 0.5f), V.Hf), tile_oy);
          }
          s.px[k][q] = ppx;
          s.py[k][q] = ppy;
        }
        s.behind[k] = behind ? 1u : 0u;
        uint32_t flips = 0u;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const int ia = kFaces[f][0], ib = kFaces[f][1], ic = kFaces[f][2], io = kFaces[f][3];
          const float e1x = fs(vx[ic], vx[ia]), e1y = fs(vy[ic], vy[ia]), e1z = fs(vz[ic], vz[ia]);
          const float e2x = fs(vx[ib], vx[ia]), e2y = fs(vy[ib], vy[ia]), e2z = fs(vz[ib], vz[ia]);
          float nx = fs(fm(e1y, e2z), fm(e1z, e2y));
          float ny = fs(fm(e1z, e2x), fm(e1x, e2z));
          float nz = fs(fm(e1x, e2y), fm(e1y, e2x));
          const float ox = fs(vx[io], vx[ia]), oy = fs(vy[io], vy[ia]), oz = fs(vz[io], vz[ia]);
          if (dot3x(nx, ny, nz, ox, oy, oz) < 0.0f) {
            nx = -nx; ny = -ny; nz = -nz;
            flips |= 1u << f;
          }
          const float num = dot3x(nx, ny, nz, fs(vx[ia], camx), fs(vy[ia], camy), fs(vz[ia], camz));
          s.nrm[k][f] = make_float4(nx, ny, nz, num);
        }
        const float gx = r.b.w, gy = r.c.w, gz = r.d.w;
        const float boff = dot3x(gx, gy, gz, fs(camx, vx[0]), fs(camy, vy[0]), fs(camz, vz[0]));
        s.cb[k] = make_float4(fa(col.x, boff), fa(col.y, boff), fa(col.z, boff), r.a.w);
        s.gr[k] = make_float4(gx, gy, gz, __uint_as_float(flips));
      }
    };
    // per-(tet,row) pixel spans, exact arithmetic.  vertex_rows selects the
    // forward rule (rasterize_compute.wgsl:170-275); without it this is the
    // adjoint rule (backward_tiled_compute.wgsl:241-299).
    auto spans = [&](int nb, bool vertex_rows) {
      for (int task = tid; task < nb * TS; task += NT) {
        const int k = task / TS, row = task - (task / TS) * TS;
        float xl = 1e10f, xr = -1e10f;
        if (!s.behind[k]) {
          const float yc = fa((float)row, 0.5f);
          const int ei[6] = {0, 0, 0, 1, 1, 2};
          const int ej[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
          for (int e = 0; e < 6; ++e) {
            const float yi = s.py[k][ei[e]], yj = s.py[k][ej[e]];
            if ((yi <= yc && yj > yc) || (yj <= yc && yi > yc)) {
              const float t = fdv(fs(yc, yi), fs(yj, yi));
              const float x = fa(s.px[k][ei[e]], fm(t, fs(s.px[k][ej[e]], s.px[k][ei[e]])));
              xl = fminf(xl, x);
              xr = fmaxf(xr, x);
            }
          }
          if (vertex_rows) {
            const float blo = fs(yc, 0.5f), bhi = fa(yc, 0.5f);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const float vyq = s.py[k][q];
              if (vyq >= blo && vyq < bhi) {
                xl = fminf(xl, s.px[k][q]);
                xr = fmaxf(xr, s.px[k][q]);
              }
            }
          }
        }
        short2 sp = make_short2(0, -1);
        if (xl <= xr) {
          const int32_t lo = max(__float2int_rz(ceilf(fs(fs(xl, 0.5f), 0.001f))), 0);
          const int32_t hi = min(__float2int_rz(floorf(fa(fs(xr, 0.5f), 0.001f))), TS - 1);
          if (lo <= hi) sp = make_short2((short)lo, (short)hi);
        }
        s.span[k][row] = sp;
      }
    };

    float Cr = 0.f, Cg = 0.f, Cb = 0.f, logT = 0.f;
    float nd0 = 0.f, nd1 = 0.f, nd2 = 0.f, nd3 = 0.f, en0 = 0.f, en1 = 0.f, en2 = 0.f, en3 = 0.f;

    // =============== forward (front to back) ===============
    if (MODE == kModeForward || MODE == kModeTrain) {
      bool alive = valid;
      if (re > rs) {
        int nb0 = (int)min((uint32_t)kBatch, re - rs);
        issue(0, re - 1u, nb0, -1);
        int b = 0;
        for (uint32_t hi = re; hi > rs;) {
          const int buf = b & 1;
          const int nb = (int)min((uint32_t)kBatch, hi - rs);
          const uint32_t next_hi = hi - (uint32_t)nb;
          wait_buf(buf);
          if (failed) break;
          if (next_hi > rs) issue(buf ^ 1, next_hi - 1u, (int)min((uint32_t)kBatch, next_hi - rs), -1);
          setup(buf, nb);
          __syncthreads();
          spans(nb, true);
          __syncthreads();
          if (alive) {
            for (int k = 0; k < nb; ++k) {
              const short2 sp = s.span[k][prow];
              if (pcol < sp.x || pcol > sp.y) continue;
              if (logT < -13.8f) { alive = false; break; }
              float t_min = -3.402823e38f, t_max = 3.402823e38f;
              int entry = 4;
              bool ok = true;
#pragma unroll
              for (int f = 0; f < 4; ++f) {
                const float4 n = s.nrm[k][f];
                const float den = dot3x(n.x, n.y, n.z, dx, dy, dz);
                const float num = has_min_t ? face_num_offset(s.rec[buf][k], f, n, ox, oy, oz) : n.w;
                if (fabsf(den) < 1e-20f) {
                  if (num > 0.0f) ok = false;
                  continue;
                }
                const float t = fdv(num, den);
                if (den > 0.0f) {
                  if (t > t_min) { t_min = t; entry = f; }
                } else {
                  if (t < t_max) t_max = t;
                }
              }
              if (!(ok && t_min < t_max)) continue;
              const float4 cb = s.cb[k];
              const float4 gg = s.gr[k];
              const float dcdt = dot3x(gg.x, gg.y, gg.z, dx, dy, dz);
              float bcr = cb.x, bcg = cb.y, bcb = cb.z;
              if (has_min_t) {  // base offset at the shifted origin, dot(g, o - v0)
                const TetRec& rr = s.rec[buf][k];
                const float bo = dot3x(gg.x, gg.y, gg.z, fs(ox, rr.a.x), fs(oy, rr.a.y), fs(oz, rr.a.z));
                const float4 cc = s.col[buf][k];
                bcr = fa(cc.x, bo); bcg = fa(cc.y, bo); bcb = fa(cc.z, bo);
              }
              const float csr = fmaxf(bcr + dcdt * t_min, 0.f), csg = fmaxf(bcg + dcdt * t_min, 0.f),
                          csb = fmaxf(bcb + dcdt * t_min, 0.f);
              const float cer = fmaxf(bcr + dcdt * t_max, 0.f), ceg = fmaxf(bcg + dcdt * t_max, 0.f),
                          ceb = fmaxf(bcb + dcdt * t_max, 0.f);
              const float dist = t_max - t_min;
              const float od = clipf(cb.w * dist, 1e-8f, 88.0f);
              const float alpha_t = __expf(-od);
              const float ph = fabsf(od) < 0.02f ? 1.0f + od * (-0.5f + od * (1.0f / 6.0f + od * (-1.0f / 24.0f)))
                                                 : clipf(__fdividef(1.0f - alpha_t, od), kMinVal, kMaxVal);
              const float w0 = ph - alpha_t, w1 = 1.0f - ph;
              const float cpr = clipf(cer * w0 + csr * w1, 0.f, kMaxVal);
              const float cpg = clipf(ceg * w0 + csg * w1, 0.f, kMaxVal);
              const float cpb = clipf(ceb * w0 + csb * w1, 0.f, kMaxVal);
              const float Tj = __expf(fmaxf(logT, -88.0f));
              if (Tj >= 1e-6f) {
                Cr += cpr * Tj; Cg += cpg * Tj; Cb += cpb * Tj;
                logT -= od;
                if (AUX) {
                  const float alpha = 1.0f - alpha_t;
                  float enx = 0.f, eny = 0.f, enz = 0.f;
                  if (entry < 4) {
                    const float4 n = s.nrm[k][entry];
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
                }
              }
            }
          }
          hi = next_hi;
          ++b;
          // all pixels saturated: the remaining tets would all be skipped
          if (__syncthreads_count(alive && logT >= -13.8f) == 0) {
            if (hi > rs) { wait_buf(buf ^ 1); }  // drain the prefetch already in flight
            break;
          }
        }
      }
      if (valid && (MODE == kModeForward || a.rgba != nullptr)) {
        const float A = 1.0f - safe_exp(logT);
        reinterpret_cast<float4*>(a.rgba)[pix] = make_float4(Cr, Cg, Cb, A);
        if (AUX && a.aux) {
          reinterpret_cast<float4*>(a.aux)[2 * pix] = make_float4(nd0, nd1, nd2, nd3);
          reinterpret_cast<float4*>(a.aux)[2 * pix + 1] = make_float4(en0, en1, en2, en3);
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
          dlogT = -0.0f * (1.0f - A);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) s.red[warp] = lsum;
        __syncthreads();
        if (tid == 0) {
          double tot = 0.0;
          for (int w = 0; w < NW; ++w) tot += (double)s.red[w];
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
      if (re > rs) {
        int nb0 = (int)min((uint32_t)kBatch, re - rs);
        __syncthreads();
        issue(0, rs, nb0, +1);
        int b = 0;
        for (uint32_t lo = rs; lo < re;) {
          const int buf = b & 1;
          const int nb = (int)min((uint32_t)kBatch, re - lo);
          const uint32_t next_lo = lo + (uint32_t)nb;
          wait_buf(buf);
          if (failed) break;
          if (next_lo < re) issue(buf ^ 1, next_lo, (int)min((uint32_t)kBatch, re - next_lo), +1);
          setup(buf, nb);
          __syncthreads();
          spans(nb, false);  // adjoint: edge crossings only
          __syncthreads();
          for (int k = 0; k < nb; ++k) {
            float c19[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) c19[q] = 0.0f;
            bool has = false;
            const short2 sp = s.span[k][prow];
            if (valid && pcol >= sp.x && pcol <= sp.y) {
              float t_min = -3.402823e38f, t_max = 3.402823e38f;
              int min_face = 0, max_face = 0;
              bool ok = true;
#pragma unroll
              for (int f = 0; f < 4; ++f) {
                const float4 n = s.nrm[k][f];
                const float den = dot3x(n.x, n.y, n.z, dx, dy, dz);
                if (fabsf(den) < 1e-20f) {
                  if (n.w > 0.0f) ok = false;
                  continue;
                }
                const float t = fdv(n.w, den);
                if (den > 0.0f) {
                  if (t > t_min) { t_min = t; min_face = f; }
                } else {
                  if (t < t_max) { t_max = t; max_face = f; }
                }
              }
              if (ok && t_min < t_max) {
                const float4 cb = s.cb[k];
                const float4 gg = s.gr[k];
                const float dens = cb.w;
                const float dcdt = dot3x(gg.x, gg.y, gg.z, dx, dy, dz);
                const float csr_r = cb.x + dcdt * t_min, csg_r = cb.y + dcdt * t_min, csb_r = cb.z + dcdt * t_min;
                const float cer_r = cb.x + dcdt * t_max, ceg_r = cb.y + dcdt * t_max, ceb_r = cb.z + dcdt * t_max;
                const float csr = fmaxf(csr_r, 0.f), csg = fmaxf(csg_r, 0.f), csb = fmaxf(csb_r, 0.f);
                const float cer = fmaxf(cer_r, 0.f), ceg = fmaxf(ceg_r, 0.f), ceb = fmaxf(ceb_r, 0.f);
                const float dist = t_max - t_min;
                const float od_raw = dens * dist;
                const float od = clipf(od_raw, 1e-8f, 88.0f);
                const float alpha_t = __expf(-od);
                const float ph = fabsf(od) < 0.02f ? 1.0f + od * (-0.5f + od * (1.0f / 6.0f + od * (-1.0f / 24.0f)))
                                                   : clipf(__fdividef(1.0f - alpha_t, od), kMinVal, kMaxVal);
                const float w0 = ph - alpha_t, w1 = 1.0f - ph;
                const float cpr = clipf(cer * w0 + csr * w1, kMinVal, kMaxVal);
                const float cpg = clipf(ceg * w0 + csg * w1, kMinVal, kMaxVal);
                const float cpb = clipf(ceb * w0 + csb * w1, kMinVal, kMaxVal);
                const float prev_logT = fminf(logT + od, 0.0f);
                const float t_prev = __expf(fmaxf(prev_logT, -88.0f));
                Cr -= cpr * t_prev; Cg -= cpg * t_prev; Cb -= cpb * t_prev;
                logT = prev_logT;
                if (t_prev >= 1e-6f) {
                  has = true;
                  const float dcpr = clipf(dlr * t_prev, kMinVal, kMaxVal);
                  const float dcpg = clipf(dlg * t_prev, kMinVal, kMaxVal);
                  const float dcpb = clipf(dlb * t_prev, kMinVal, kMaxVal);
                  const float d_od_state = -dlogT;
                  dlogT = clipf(dlogT + (dlr * cpr + dlg * cpg + dlb * cpb) * t_prev, kMinVal, kMaxVal);
                  float dph;
                  if (fabsf(od) < 0.02f) dph = -0.5f + od * (1.0f / 3.0f + od * (-1.0f / 8.0f + od * (1.0f / 30.0f)));
                  else dph = clipf(__fdividef(alpha_t * (od + 1.0f) - 1.0f, od * od), kMinVal, kMaxVal);
                  const float dw0 = dph + alpha_t, dw1 = -dph;
                  const float d_od_int = dcpr * (cer * dw0 + csr * dw1) + dcpg * (ceg * dw0 + csg * dw1) +
                                         dcpb * (ceb * dw0 + csb * dw1);
                  const float d_od = clipf(d_od_state + d_od_int, kMinVal, kMaxVal);
                  const bool active = (od_raw >= 1e-8f) && (od_raw <= 88.0f);
                  const float d_od_raw = active ? d_od : 0.0f;
                  const float d_dens = clipf(d_od_raw * dist, kMinVal, kMaxVal);
                  const float d_dist = clipf(d_od_raw * dens, kMinVal, kMaxVal);
                  float d_tmin = -d_dist, d_tmax = d_dist;
                  const float dsr = csr_r > 0.f ? dcpr * w1 : 0.f, dsg = csg_r > 0.f ? dcpg * w1 : 0.f,
                              dsb = csb_r > 0.f ? dcpb * w1 : 0.f;
                  const float der = cer_r > 0.f ? dcpr * w0 : 0.f, deg = ceg_r > 0.f ? dcpg * w0 : 0.f,
                              deb = ceb_r > 0.f ? dcpb * w0 : 0.f;
                  const float dbr = dsr + der, dbg = dsg + deg, dbb = dsb + deb;
                  const float ss = dsr + dsg + dsb, se = der + deg + deb;
                  const float d_dcdt = ss * t_min + se * t_max;
                  d_tmin += ss * dcdt;
                  d_tmax += se * dcdt;
                  const float sb = dbr + dbg + dbb;
                  const TetRec& r = s.rec[buf][k];
                  const float vx[4] = {r.a.x, r.b.x, r.c.x, r.d.x};
                  const float vy[4] = {r.a.y, r.b.y, r.c.y, r.d.y};
                  const float vz[4] = {r.a.z, r.b.z, r.c.z, r.d.z};
                  c19[0] = clipf(d_dens, kMinVal, kMaxVal);
                  c19[1] = clipf(dbr, kMinVal, kMaxVal);
                  c19[2] = clipf(dbg, kMinVal, kMaxVal);
                  c19[3] = clipf(dbb, kMinVal, kMaxVal);
                  c19[4] = clipf((camx - vx[0]) * sb + dx * d_dcdt, kMinVal, kMaxVal);
                  c19[5] = clipf((camy - vy[0]) * sb + dy * d_dcdt, kMinVal, kMaxVal);
                  c19[6] = clipf((camz - vz[0]) * sb + dz * d_dcdt, kMinVal, kMaxVal);
                  float dv[12];
#pragma unroll
                  for (int q = 0; q < 12; ++q) dv[q] = 0.0f;
                  const uint32_t flips = __float_as_uint(gg.w);
#pragma unroll
                  for (int side = 0; side < 2; ++side) {
                    const int f = side == 0 ? min_face : max_face;
                    const float dt = side == 0 ? d_tmin : d_tmax;
                    const float tt = side == 0 ? t_min : t_max;
                    const int ia = kFaces[f][0], ib = kFaces[f][1], ic = kFaces[f][2];
                    const float4 nf = s.nrm[k][f];
                    const float sg = ((flips >> f) & 1u) ? -1.0f : 1.0f;  // undo the inward flip
                    const float nx = sg * nf.x, ny = sg * nf.y, nz = sg * nf.z;
                    const float den = nx * dx + ny * dy + nz * dz;
                    const float inv_den = fabsf(den) < kTiny ? clipf(1.0f / kTiny, kMinVal, kMaxVal)
                                                             : clipf(1.0f / den, kMinVal, kMaxVal);
                    const float hx = camx + dx * tt, hy = camy + dy * tt, hz = camz + dz * tt;
                    const float ahx = vx[ia] - hx, ahy = vy[ia] - hy, ahz = vz[ia] - hz;
                    // dt/dva = (cross(va-hit, vb-vc) + n) / den
                    float ux = vx[ib] - vx[ic], uy = vy[ib] - vy[ic], uz = vz[ib] - vz[ic];
                    float gax = (ahy * uz - ahz * uy + nx) * inv_den, gay = (ahz * ux - ahx * uz + ny) * inv_den,
                          gaz = (ahx * uy - ahy * ux + nz) * inv_den;
                    // dt/dvb = cross(va-hit, vc-va) / den
                    ux = vx[ic] - vx[ia]; uy = vy[ic] - vy[ia]; uz = vz[ic] - vz[ia];
                    float gbx = (ahy * uz - ahz * uy) * inv_den, gby = (ahz * ux - ahx * uz) * inv_den,
                          gbz = (ahx * uy - ahy * ux) * inv_den;
                    // dt/dvc = cross(va-hit, va-vb) / den
                    ux = vx[ia] - vx[ib]; uy = vy[ia] - vy[ib]; uz = vz[ia] - vz[ib];
                    float gcx = (ahy * uz - ahz * uy) * inv_den, gcy = (ahz * ux - ahx * uz) * inv_den,
                          gcz = (ahx * uy - ahy * ux) * inv_den;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                      if (q == ia) {
                        dv[3 * q] += clipf(gax * dt, kMinVal, kMaxVal);
                        dv[3 * q + 1] += clipf(gay * dt, kMinVal, kMaxVal);
                        dv[3 * q + 2] += clipf(gaz * dt, kMinVal, kMaxVal);
                      } else if (q == ib) {
                        dv[3 * q] += clipf(gbx * dt, kMinVal, kMaxVal);
                        dv[3 * q + 1] += clipf(gby * dt, kMinVal, kMaxVal);
                        dv[3 * q + 2] += clipf(gbz * dt, kMinVal, kMaxVal);
                      } else if (q == ic) {
                        dv[3 * q] += clipf(gcx * dt, kMinVal, kMaxVal);
                        dv[3 * q + 1] += clipf(gcy * dt, kMinVal, kMaxVal);
                        dv[3 * q + 2] += clipf(gcz * dt, kMinVal, kMaxVal);
                      }
                    }
                  }
                  dv[0] += -gg.x * sb;
                  dv[1] += -gg.y * sb;
                  dv[2] += -gg.z * sb;
#pragma unroll
                  for (int q = 0; q < 12; ++q) c19[7 + q] = clipf(dv[q], kMinVal, kMaxVal);
                }
              }
            }
            const unsigned m = __ballot_sync(0xffffffffu, has);
            if (m) {
              float* acc = reinterpret_cast<float*>(&s.acc[k][0]);
              if (__popc(m) <= 2) {
                if (has) {
#pragma unroll
                  for (int q = 0; q < 19; ++q) atomicAdd(&acc[q], c19[q]);
                }
              } else {
                const float r = warp_reduce_scatter<19>(c19, lane);
                if (lane < 19) atomicAdd(&acc[lane], r);
              }
            }
          }
          __syncthreads();
          // flush this batch's per-tet sums (five 16-byte vector atomics per tet)
          for (int q = tid; q < nb * 5; q += NT) {
            const int k = q / 5, c = q - (q / 5) * 5;
            const float4 v4 = s.acc[k][c];
            if (v4.x != 0.f || v4.y != 0.f || v4.z != 0.f || v4.w != 0.f) {
              atomicAdd(reinterpret_cast<float4*>(a.grad_slot + (size_t)s.tet[buf][k] * kGradSlot) + c, v4);
              s.acc[k][c] = make_float4(0.f, 0.f, 0.f, 0.f);
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

}  // namespace rm
