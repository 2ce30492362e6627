/*
 * rmesh_oracle.c -- CPU restatement of the rmeshvk tiled volume-rendering path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * is compared against; it is never linked into the product library.  Only the
 * test tree, the smoke check and the CPU-baseline leg of the benchmark load it.
 *
 * It restates, function by function, the WGSL kernels of the reference
 * (paths relative to the reference repository root):
 *
 *   orc_project      crates/rmesh-render/src/wgsl/project_compute.wgsl:88-325
 *   orc_emit         crates/rmesh-tile/src/wgsl/tile_gen_scan_compute.wgsl:61-203
 *                    (slots a tet cannot fill keep the sentinel written by
 *                    crates/rmesh-tile/src/wgsl/tile_fill_compute.wgsl:9-19)
 *   orc_sort_pairs   crates/rmesh-sort/src/drs.rs:23-26,180-279 (stable LSD sort of
 *                    the low `sorting_bits` bits of the 64-bit (tile, ~depth) key)
 *   orc_tile_ranges  crates/rmesh-tile/src/wgsl/tile_ranges_compute.wgsl:10-45
 *   orc_rasterize    crates/rmesh-render/src/wgsl/rasterize_compute.wgsl:92-511
 *   orc_loss         crates/rmesh-train/src/wgsl/loss_compute.wgsl:24-72
 *   orc_backward     crates/rmesh-backward/src/wgsl/backward_tiled_compute.wgsl:154-587
 *   orc_adam         crates/rmesh-train/src/wgsl/adam_compute.wgsl:121-149
 *   math helpers     crates/rmesh-util/src/wgsl/math.wgsl:1-71,
 *                    crates/rmesh-util/src/wgsl/intersect.wgsl:4-10
 *
 * Canonical order: the reference compacts visible tets with atomicAdd
 * (project_compute.wgsl:181), so its pre-sort pair order is run-to-run
 * nondeterministic.  The oracle emits tets in tet-id order, which makes the
 * stable sort break key ties by tet index.
 *
 * Float semantics: compiled with -ffp-contract=off so every WGSL multiply and
 * add is a separately rounded IEEE single operation, evaluated left to right
 * (dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z; mat*vec = ((c0*x + c1*y) + c2*z) + c3*w).
 * WGSL's f32->u32 / f32->i32 conversions saturate; f2u/f2i below do the same.
 *
 * The same source is compiled twice: REAL=float (symbols *_f32) for parity and
 * REAL=double (symbols *_f64) for finite-difference gradient checks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_DOUBLE
typedef double R;
#define SFX(name) name##_f64
#define RSQRT(x) sqrt(x)
#define REXP(x) exp(x)
#define RLOG(x) log(x)
#define RFLOOR(x) floor(x)
#define RCEIL(x) ceil(x)
#define RMIN(a, b) fmin(a, b)
#define RMAX(a, b) fmax(a, b)
#define RABS(x) fabs(x)
#else
typedef float R;
#define SFX(name) name##_f32
#define RSQRT(x) sqrtf(x)
#define REXP(x) expf(x)
#define RLOG(x) logf(x)
#define RFLOOR(x) floorf(x)
#define RCEIL(x) ceilf(x)
#define RMIN(a, b) fminf(a, b)
#define RMAX(a, b) fmaxf(a, b)
#define RABS(x) fabsf(x)
#endif

#define EXPORT __attribute__((visibility("default")))

/* ---- safe math (math.wgsl:3-65) ---------------------------------------- */
static const R TINY_VAL = (R)1.0754944e-20;
static const R MIN_VAL = (R)-1e+20;
static const R MAX_VAL = (R)1e+20;
static const R LOG_MAX_VAL = (R)46.0517;

static inline R clipr(R v, R lo, R hi) { return RMAX(RMIN(v, hi), lo); }
static inline R safe_div(R a, R b) {
    if (RABS(b) < TINY_VAL) return clipr(a / TINY_VAL, MIN_VAL, MAX_VAL);
    return clipr(a / b, MIN_VAL, MAX_VAL);
}
static inline R safe_exp(R v) { return REXP(clipr(v, (R)-88.0, LOG_MAX_VAL)); }
static inline R safe_sqrt(R a) { return a < TINY_VAL ? (R)0 : RSQRT(a); }
static inline R phi(R x) {
    if (RABS(x) < (R)0.02)
        return (R)1 + x * ((R)-0.5 + x * ((R)1 / (R)6 + x * ((R)-1 / (R)24)));
    return safe_div((R)1 - REXP(-x), x);
}
static inline R dphi_dx(R x) {
    if (RABS(x) < (R)0.02)
        return (R)-0.5 + x * ((R)1 / (R)3 + x * ((R)-1 / (R)8 + x * ((R)1 / (R)30)));
    R ex = REXP(-x);
    return safe_div(ex * (x + (R)1) - (R)1, x * x);
}
static inline R softplus(R x) {
    if (x * (R)10 > (R)20) return x;
    return (R)0.1 * RLOG((R)1 + REXP((R)10 * x));
}

/* WGSL u32(f32) / i32(f32): saturating, NaN -> 0. */
static inline uint32_t f2u(R x) {
    if (!(x > (R)0)) return 0u;
    if (x >= (R)4294967296.0) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
static inline int32_t f2i(R x) {
    if (x != x) return 0;
    if (x >= (R)2147483648.0) return INT32_MAX;
    if (x <= (R)-2147483648.0) return INT32_MIN;
    return (int32_t)x;
}

/* ---- vec3 helpers (left-to-right evaluation) ----------------------------- */
typedef struct { R x, y, z; } V3;
static inline V3 v3(R x, R y, R z) { V3 r = {x, y, z}; return r; }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vscale(V3 a, R s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline R vdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline V3 vnormalize(V3 a) {
    R l = RSQRT(vdot(a, a));
    return v3(a.x / l, a.y / l, a.z / l);
}
static inline V3 vclip(V3 a, R lo, R hi) { return v3(clipr(a.x, lo, hi), clipr(a.y, lo, hi), clipr(a.z, lo, hi)); }
static inline V3 vmax0(V3 a) { return v3(RMAX(a.x, (R)0), RMAX(a.y, (R)0), RMAX(a.z, (R)0)); }

static inline V3 load_v3(const R* p, uint32_t i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

/* clip = vp * vec4(v, 1), vp column-major (vp[col*4+row]). */
static inline void mat4_mul_point(const R* vp, V3 v, R out[4]) {
    for (int r = 0; r < 4; ++r)
        out[r] = ((vp[0 * 4 + r] * v.x + vp[1 * 4 + r] * v.y) + vp[2 * 4 + r] * v.z) + vp[3 * 4 + r];
}
/* c2w * v, c2w column-major 3x3 (c2w[col*3+row]). */
static inline V3 mat3_mul(const R* c2w, V3 v) {
    R o[3];
    for (int r = 0; r < 3; ++r) o[r] = (c2w[0 * 3 + r] * v.x + c2w[1 * 3 + r] * v.y) + c2w[2 * 3 + r] * v.z;
    return v3(o[0], o[1], o[2]);
}

/* FACES (intersect.wgsl:4-10): (a, b, c, opposite). */
static const int FACES[4][4] = {{0, 2, 1, 3}, {1, 2, 3, 0}, {0, 3, 2, 1}, {3, 0, 1, 2}};
static const int EI[6] = {0, 0, 0, 1, 1, 2};
static const int EJ[6] = {1, 2, 3, 2, 3, 3};

/* SH constants (project_compute.wgsl:51-64). */
static const R C0 = (R)0.28209479177387814;
static const R C1 = (R)0.4886025119029199;
static const R C2_0 = (R)1.0925484305920792, C2_1 = (R)-1.0925484305920792, C2_2 = (R)0.31539156525252005,
               C2_3 = (R)-1.0925484305920792, C2_4 = (R)0.5462742152960396;
static const R C3_0 = (R)-0.5900435899266435, C3_1 = (R)2.890611442640554, C3_2 = (R)-0.4570457994644658,
               C3_3 = (R)0.3731763325901154, C3_4 = (R)-0.4570457994644658, C3_5 = (R)1.445305721320277,
               C3_6 = (R)-0.5900435899266435;

/* SH basis value i at unit direction (x, y, z), as the reference evaluates it
 * term by term (project_compute.wgsl:282-305): the coefficient multiplies the
 * product of the constant and the direction monomial. */
static inline R sh_basis(uint32_t i, R x, R y, R z) {
    R xx = x * x, yy = y * y, zz = z * z;
    switch (i) {
        case 0: return C0;
        case 1: return -(C1 * y);
        case 2: return C1 * z;
        case 3: return -(C1 * x);
        case 4: return C2_0 * (x * y);
        case 5: return C2_1 * (y * z);
        case 6: return C2_2 * ((R)2 * zz - xx - yy);
        case 7: return C2_3 * (x * z);
        case 8: return C2_4 * (xx - yy);
        case 9: return C3_0 * y * ((R)3 * xx - yy);
        case 10: return C3_1 * x * y * z;
        case 11: return C3_2 * y * ((R)4 * zz - xx - yy);
        case 12: return C3_3 * z * ((R)2 * zz - (R)3 * xx - (R)3 * yy);
        case 13: return C3_4 * x * ((R)4 * zz - xx - yy);
        case 14: return C3_5 * z * (xx - yy);
        default: return C3_6 * x * (xx - (R)3 * yy);
    }
}

/* d basis_i / d(x, y, z), direction components treated as independent. */
static inline V3 sh_basis_grad(uint32_t i, R x, R y, R z) {
    R xx = x * x, yy = y * y, zz = z * z;
    switch (i) {
        case 0: return v3(0, 0, 0);
        case 1: return v3(0, -C1, 0);
        case 2: return v3(0, 0, C1);
        case 3: return v3(-C1, 0, 0);
        case 4: return v3(C2_0 * y, C2_0 * x, 0);
        case 5: return v3(0, C2_1 * z, C2_1 * y);
        case 6: return v3(-(R)2 * C2_2 * x, -(R)2 * C2_2 * y, (R)4 * C2_2 * z);
        case 7: return v3(C2_3 * z, 0, C2_3 * x);
        case 8: return v3((R)2 * C2_4 * x, -(R)2 * C2_4 * y, 0);
        case 9: return v3((R)6 * C3_0 * x * y, C3_0 * ((R)3 * xx - (R)3 * yy), 0);
        case 10: return v3(C3_1 * y * z, C3_1 * x * z, C3_1 * x * y);
        case 11: return v3(-(R)2 * C3_2 * x * y, C3_2 * ((R)4 * zz - xx - (R)3 * yy), (R)8 * C3_2 * y * z);
        case 12: return v3(-(R)6 * C3_3 * x * z, -(R)6 * C3_3 * y * z, C3_3 * ((R)6 * zz - (R)3 * xx - (R)3 * yy));
        case 13: return v3(C3_4 * ((R)4 * zz - (R)3 * xx - yy), -(R)2 * C3_4 * x * y, (R)8 * C3_4 * x * z);
        case 14: return v3((R)2 * C3_5 * x * z, -(R)2 * C3_5 * y * z, C3_5 * (xx - yy));
        default: return v3(C3_6 * ((R)3 * xx - (R)3 * yy), -(R)6 * C3_6 * x * y, 0);
    }
}

/* d softplus(x) / dx (crates/rmesh-util/src/wgsl/math.wgsl:27-33). */
static inline R dsoftplus(R x) {
    if (x * (R)10 > (R)20) return (R)1;
    R e = REXP((R)10 * x);
    return safe_div(e, (R)1 + e);
}

/* Unit direction from the camera to the tet centroid and the centroid itself
 * (project_compute.wgsl:268-273). */
static inline R sh_dir(const V3 v[4], const R* cam3, V3* centroid, V3* dir) {
    *centroid = vscale(vadd(vadd(vadd(v[0], v[1]), v[2]), v[3]), (R)0.25);
    V3 raw = vsub(*centroid, v3(cam3[0], cam3[1], cam3[2]));
    R len = RSQRT(vdot(raw, raw));
    *dir = v3(0, 0, 0);
    if (len > (R)0) *dir = v3(raw.x / len, raw.y / len, raw.z / len);
    return len;
}

/* ======================================================================== */
/* orc_project -- project_compute.wgsl:88-325 (per tet id).                 */
/* Outputs, indexed by tet id: visible (0/1), tiles_touched, colors[3M].    */
/* sh == NULL selects the base_colors copy branch (:319-324).  sh holds the  */
/* coefficient values [M][3][nc] the shader reads: the reference stores    */
/* them as f16 (crates/rmesh-viewer/src/gpu_state.rs:60-88), so callers    */
/* pass f16-rounded values for parity and unrounded ones for f64 checks.  */
/* ======================================================================== */
static void project_one(uint32_t t, const R* verts, const uint32_t* idx, const R* dens, const R* cgrad,
                        const R* circ, const R* base, const R* sh, int sh_degree, const R* vp,
                        const R* cam3, R W, R H, uint32_t ts, uint8_t* visible, uint32_t* tiles_touched,
                        R* colors) {
    (void)circ;
    V3 v[4];
    for (int k = 0; k < 4; ++k) v[k] = load_v3(verts, idx[4 * t + k]);
    R p[4][4];
    for (int k = 0; k < 4; ++k) {
        R c[4];
        mat4_mul_point(vp, v[k], c);
        R inv_w = (R)1 / (c[3] + (R)1e-6);
        p[k][0] = c[0] * inv_w; p[k][1] = c[1] * inv_w; p[k][2] = c[2] * inv_w; p[k][3] = c[3];
    }
    int any_behind = (p[0][3] <= 0) || (p[1][3] <= 0) || (p[2][3] <= 0) || (p[3][3] <= 0);
    int vis = 1;
    if (!any_behind) {
        R min_x = RMIN(RMIN(p[0][0], p[1][0]), RMIN(p[2][0], p[3][0]));
        R max_x = RMAX(RMAX(p[0][0], p[1][0]), RMAX(p[2][0], p[3][0]));
        R min_y = RMIN(RMIN(p[0][1], p[1][1]), RMIN(p[2][1], p[3][1]));
        R max_y = RMAX(RMAX(p[0][1], p[1][1]), RMAX(p[2][1], p[3][1]));
        R min_z = RMIN(RMIN(p[0][2], p[1][2]), RMIN(p[2][2], p[3][2]));
        if (max_x < (R)-1 || min_x > (R)1 || max_y < (R)-1 || min_y > (R)1 || min_z > (R)1) vis = 0;
        R ext_x = (max_x - min_x) * W;
        R ext_y = (max_y - min_y) * H;
        if (ext_x * ext_y < (R)1) vis = 0;
    }
    visible[t] = 0;
    tiles_touched[t] = 0;
    if (!vis) return;
    {
        V3 e01 = vsub(v[1], v[0]), e02 = vsub(v[2], v[0]), e03 = vsub(v[3], v[0]);
        V3 e12 = vsub(v[2], v[1]), e13 = vsub(v[3], v[1]), e23 = vsub(v[3], v[2]);
        R m = RMAX(RMAX(vdot(e01, e01), RMAX(vdot(e02, e02), vdot(e03, e03))),
                   RMAX(vdot(e12, e12), RMAX(vdot(e13, e13), vdot(e23, e23))));
        R max_od = dens[t] * RSQRT(m);
        if (max_od < (R)0.01) return;
    }
    visible[t] = 1;
    uint32_t count = 0;
    if (!any_behind) {
        R px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            px[k] = (p[k][0] + (R)1) * (R)0.5 * W;
            py[k] = ((R)1 - p[k][1]) * (R)0.5 * H;
        }
        R pix_min_x = RMAX(RMIN(RMIN(px[0], px[1]), RMIN(px[2], px[3])), (R)0);
        R pix_max_x = RMIN(RMAX(RMAX(px[0], px[1]), RMAX(px[2], px[3])), W - (R)1);
        R pix_min_y = RMAX(RMIN(RMIN(py[0], py[1]), RMIN(py[2], py[3])), (R)0);
        R pix_max_y = RMIN(RMAX(RMAX(py[0], py[1]), RMAX(py[2], py[3])), H - (R)1);
        if (!(pix_min_x > pix_max_x || pix_min_y > pix_max_y)) {
            R T = (R)ts;
            uint32_t tiles_x_total = f2u(RCEIL(W / T));
            uint32_t tile_min_x = f2u(pix_min_x / T);
            uint32_t tile_max_x = f2u(pix_max_x / T);
            if (tile_max_x > tiles_x_total - 1u) tile_max_x = tiles_x_total - 1u;
            uint32_t tile_min_y = f2u(pix_min_y / T);
            uint32_t tile_max_y = f2u(pix_max_y / T);
            uint32_t tyt = f2u(RCEIL(H / T)) - 1u;
            if (tile_max_y > tyt) tile_max_y = tyt;
            for (uint32_t ty = tile_min_y; ty <= tile_max_y; ++ty) {
                R xl = (R)1e10, xr = (R)-1e10;
                for (int e = 0; e < 6; ++e) {
                    R yi = py[EI[e]], yj = py[EJ[e]], xi = px[EI[e]], xj = px[EJ[e]];
                    for (uint32_t b = 0; b < 2; ++b) {
                        R ytest = (R)(ty + b) * T;
                        if ((yi <= ytest && yj > ytest) || (yj <= ytest && yi > ytest)) {
                            R tt = (ytest - yi) / (yj - yi);
                            R x = xi + tt * (xj - xi);
                            xl = RMIN(xl, x);
                            xr = RMAX(xr, x);
                        }
                    }
                }
                for (int k = 0; k < 4; ++k) {
                    R vy = py[k];
                    if (vy >= (R)ty * T && vy <= (R)(ty + 1u) * T) {
                        xl = RMIN(xl, px[k]);
                        xr = RMAX(xr, px[k]);
                    }
                }
                if (xl <= xr) {
                    uint32_t tx0 = f2u(RMAX(RFLOOR(xl / T), (R)0));
                    uint32_t tx1 = f2u(RMAX(RFLOOR(xr / T), (R)0));
                    tx0 = tx0 < tile_min_x ? tile_min_x : (tx0 > tile_max_x ? tile_max_x : tx0);
                    tx1 = tx1 < tile_min_x ? tile_min_x : (tx1 > tile_max_x ? tile_max_x : tx1);
                    count += tx1 - tx0 + 1u;
                }
            }
        }
    }
    tiles_touched[t] = count;

    /* colors (project_compute.wgsl:264-324) */
    if (sh != NULL) {
        V3 centroid, dir;
        sh_dir(v, cam3, &centroid, &dir);
        R x = dir.x, y = dir.y, z = dir.z;
        uint32_t deg = (uint32_t)sh_degree;
        uint32_t nc = (deg + 1u) * (deg + 1u);
        const R* co = sh + (size_t)t * 3u * nc;
        R rgb[3];
        for (uint32_t c = 0; c < 3; ++c) {
            const R* q = co + c * nc;
            R val = C0 * q[0];
            if (deg >= 1u) {
                val -= C1 * y * q[1];
                val += C1 * z * q[2];
                val -= C1 * x * q[3];
            }
            if (deg >= 2u) {
                R xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
                val += C2_0 * xy * q[4];
                val += C2_1 * yz * q[5];
                val += C2_2 * ((R)2 * zz - xx - yy) * q[6];
                val += C2_3 * xz * q[7];
                val += C2_4 * (xx - yy) * q[8];
            }
            if (deg >= 3u) {
                R xx = x * x, yy = y * y, zz = z * z;
                val += C3_0 * y * ((R)3 * xx - yy) * q[9];
                val += C3_1 * x * y * z * q[10];
                val += C3_2 * y * ((R)4 * zz - xx - yy) * q[11];
                val += C3_3 * z * ((R)2 * zz - (R)3 * xx - (R)3 * yy) * q[12];
                val += C3_4 * x * ((R)4 * zz - xx - yy) * q[13];
                val += C3_5 * z * (xx - yy) * q[14];
                val += C3_6 * x * (xx - (R)3 * yy) * q[15];
            }
            rgb[c] = val + (R)0.5;
        }
        V3 g = load_v3(cgrad, t);
        R off = vdot(g, vsub(v[0], centroid));
        for (int c = 0; c < 3; ++c) colors[3 * t + c] = softplus(rgb[c] + off);
    } else {
        for (int c = 0; c < 3; ++c) colors[3 * t + c] = base[3 * t + c];
    }
}

EXPORT int SFX(orc_project)(int64_t M, const R* verts, const uint32_t* idx, const R* dens, const R* cgrad,
                            const R* circ, const R* base, const R* sh, int sh_degree,
                            const R* vp, const R* cam, int W, int H, int tile_size, uint8_t* visible,
                            uint32_t* tiles_touched, R* colors) {
    R Wf = (R)W, Hf = (R)H;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < M; ++t)
        project_one((uint32_t)t, verts, idx, dens, cgrad, circ, base, sh, sh_degree, vp, cam, Wf, Hf,
                    (uint32_t)tile_size, visible, tiles_touched, colors);
    return 0;
}

/* ======================================================================== */
/* orc_emit -- tile_gen_scan_compute.wgsl:61-203 over visible tets in tet   */
/* id order.  Slot ranges come from the prefix sum of tiles_touched.        */
/* Slots a tet does not fill keep the sentinel (0xFFFFFFFF, 0xFFFFFFFF, 0). */
/* Returns P = sum of tiles_touched over visible tets; *emitted counts the  */
/* slots actually written.                                                  */
/* ======================================================================== */
EXPORT int64_t SFX(orc_emit)(int64_t M, const R* verts, const uint32_t* idx, const R* circ, const R* vp,
                             const R* cam3, int W, int H, int tile_size, const uint8_t* visible,
                             const uint32_t* tiles_touched, uint32_t* key_lo, uint32_t* key_hi,
                             uint32_t* vals, int64_t cap, int64_t* emitted) {
    int64_t* offs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(M + 1));
    int64_t acc = 0;
    for (int64_t t = 0; t < M; ++t) {
        offs[t] = acc;
        if (visible[t]) acc += tiles_touched[t];
    }
    offs[M] = acc;
    int64_t P = acc;
    for (int64_t i = 0; i < P && i < cap; ++i) { key_lo[i] = 0xFFFFFFFFu; key_hi[i] = 0xFFFFFFFFu; vals[i] = 0u; }
    R Wf = (R)W, Hf = (R)H, ts = (R)tile_size;
    uint32_t tiles_x = (uint32_t)((W + tile_size - 1) / tile_size);
    int64_t n_written = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : n_written)
    for (int64_t t = 0; t < M; ++t) {
        if (!visible[t]) continue;
        uint32_t max_write = tiles_touched[t];
        if (max_write == 0u) continue;
        int64_t write_start = offs[t];
        V3 v[4];
        for (int k = 0; k < 4; ++k) v[k] = load_v3(verts, idx[4 * t + k]);
        R px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            R c[4];
            mat4_mul_point(vp, v[k], c);
            R w = c[3] + (R)1e-6;
            R nx = c[0] / w, ny = c[1] / w;
            px[k] = (nx + (R)1) * (R)0.5 * Wf;
            py[k] = ((R)1 - ny) * (R)0.5 * Hf;
        }
        R pix_min_x = RMAX(RMIN(RMIN(px[0], px[1]), RMIN(px[2], px[3])), (R)0);
        R pix_max_x = RMIN(RMAX(RMAX(px[0], px[1]), RMAX(px[2], px[3])), Wf - (R)1);
        R pix_min_y = RMAX(RMIN(RMIN(py[0], py[1]), RMIN(py[2], py[3])), (R)0);
        R pix_max_y = RMIN(RMAX(RMAX(py[0], py[1]), RMAX(py[2], py[3])), Hf - (R)1);
        if (pix_min_x > pix_max_x || pix_min_y > pix_max_y) continue;
        uint32_t tiles_x_total = f2u(RCEIL(Wf / ts));
        uint32_t tile_min_x = f2u(pix_min_x / ts);
        uint32_t tile_max_x = f2u(pix_max_x / ts);
        if (tile_max_x > tiles_x_total - 1u) tile_max_x = tiles_x_total - 1u;
        uint32_t tile_min_y = f2u(pix_min_y / ts);
        uint32_t tile_max_y = f2u(pix_max_y / ts);
        uint32_t tyt = f2u(RCEIL(Hf / ts)) - 1u;
        if (tile_max_y > tyt) tile_max_y = tyt;
        V3 C = v3(circ[4 * t], circ[4 * t + 1], circ[4 * t + 2]);
        R r2 = circ[4 * t + 3];
        V3 diff = vsub(C, v3(cam3[0], cam3[1], cam3[2]));
        float depth = (float)(vdot(diff, diff) - r2);
        uint32_t bits;
        memcpy(&bits, &depth, 4);
        uint32_t inv_depth = ~bits;
        uint32_t local = 0;
        for (uint32_t ty = tile_min_y; ty <= tile_max_y; ++ty) {
            R xl = (R)1e10, xr = (R)-1e10;
            for (int e = 0; e < 6; ++e) {
                R yi = py[EI[e]], yj = py[EJ[e]], xi = px[EI[e]], xj = px[EJ[e]];
                for (uint32_t b = 0; b < 2; ++b) {
                    R ytest = (R)(ty + b) * ts;
                    if ((yi <= ytest && yj > ytest) || (yj <= ytest && yi > ytest)) {
                        R tt = (ytest - yi) / (yj - yi);
                        R x = xi + tt * (xj - xi);
                        xl = RMIN(xl, x);
                        xr = RMAX(xr, x);
                    }
                }
            }
            for (int k = 0; k < 4; ++k) {
                R vy = py[k];
                if (vy >= (R)ty * ts && vy <= (R)(ty + 1u) * ts) {
                    xl = RMIN(xl, px[k]);
                    xr = RMAX(xr, px[k]);
                }
            }
            if (xl <= xr) {
                uint32_t tx0 = f2u(RMAX(RFLOOR(xl / ts), (R)0));
                uint32_t tx1 = f2u(RMAX(RFLOOR(xr / ts), (R)0));
                tx0 = tx0 < tile_min_x ? tile_min_x : (tx0 > tile_max_x ? tile_max_x : tx0);
                tx1 = tx1 < tile_min_x ? tile_min_x : (tx1 > tile_max_x ? tile_max_x : tx1);
                for (uint32_t tx = tx0; tx <= tx1; ++tx) {
                    if (local < max_write) {
                        int64_t w = write_start + local;
                        if (w < cap) {
                            key_lo[w] = inv_depth;
                            key_hi[w] = ty * tiles_x + tx;
                            vals[w] = (uint32_t)t;
                            n_written++;
                        }
                        local++;
                    }
                }
            }
        }
    }
    free(offs);
    if (emitted) *emitted = n_written;
    return P;
}

/* ======================================================================== */
/* orc_sort_pairs -- the DRS sort: stable ascending on the low sorting_bits */
/* of key = (hi << 32) | lo (drs.rs:23-26; 8-bit LSD passes are stable).    */
/* ======================================================================== */
typedef struct { uint64_t k; uint64_t seq; uint32_t lo, hi, v; } SortItem;
static int cmp_item(const void* a, const void* b) {
    const SortItem* x = (const SortItem*)a;
    const SortItem* y = (const SortItem*)b;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    return x->seq < y->seq ? -1 : (x->seq > y->seq ? 1 : 0);
}
EXPORT void SFX(orc_sort_pairs)(int64_t P, int sorting_bits, uint32_t* key_lo, uint32_t* key_hi, uint32_t* vals) {
    uint64_t mask = sorting_bits >= 64 ? ~0ull : ((1ull << sorting_bits) - 1ull);
    SortItem* it = (SortItem*)malloc(sizeof(SortItem) * (size_t)(P > 0 ? P : 1));
    for (int64_t i = 0; i < P; ++i) {
        it[i].k = (((uint64_t)key_hi[i] << 32) | key_lo[i]) & mask;
        it[i].seq = (uint64_t)i;
        it[i].lo = key_lo[i]; it[i].hi = key_hi[i]; it[i].v = vals[i];
    }
    qsort(it, (size_t)P, sizeof(SortItem), cmp_item);
    for (int64_t i = 0; i < P; ++i) { key_lo[i] = it[i].lo; key_hi[i] = it[i].hi; vals[i] = it[i].v; }
    free(it);
}

/* drs.rs:23-26 */
EXPORT int SFX(orc_sorting_bits)(uint32_t num_tiles) {
    uint32_t tile_bits = num_tiles <= 1 ? 1u : 32u - (uint32_t)__builtin_clz(num_tiles - 1u);
    return (int)((32u + tile_bits + 7u) & ~7u);
}

/* ======================================================================== */
/* orc_tile_ranges -- tile_ranges_compute.wgsl:10-45, one iteration per    */
/* pair index in [0, P).  ranges must be zeroed by the caller.             */
/* ======================================================================== */
EXPORT void SFX(orc_tile_ranges)(int64_t P, const uint32_t* key_hi, uint32_t* ranges) {
    for (int64_t idx = 0; idx < P; ++idx) {
        uint32_t tile_id = key_hi[idx];
        if (tile_id == 0xFFFFFFFFu) continue;
        if (idx == 0) ranges[2u * tile_id] = (uint32_t)idx;
        else {
            uint32_t prev = key_hi[idx - 1];
            if (tile_id != prev) {
                ranges[2u * tile_id] = (uint32_t)idx;
                if (prev != 0xFFFFFFFFu) ranges[2u * prev + 1u] = (uint32_t)idx;
            }
        }
        if (idx == P - 1) ranges[2u * tile_id + 1u] = (uint32_t)(idx + 1);
    }
}

/* ---- camera description shared by the rasterizer and the adjoint ------- */
typedef struct {
    const R* vp;   /* 16, column-major */
    const R* c2w;  /* 9, column-major */
    const R* intr; /* fx, fy, cx, cy */
    const R* cam;  /* 3 */
    int W, H, TS;
    R min_t;
} Cam;

static inline V3 pixel_dir(const Cam* c, uint32_t px, uint32_t py) {
    V3 dc = v3(((R)px + (R)0.5 - c->intr[2]) / c->intr[0], ((R)py + (R)0.5 - c->intr[3]) / c->intr[1], (R)1);
    dc = vnormalize(dc);
    return vnormalize(mat3_mul(c->c2w, dc));
}

/* tile-local projected coords; returns any_behind (rasterize_compute.wgsl:152-167) */
static int tile_proj(const Cam* c, const V3 v[4], R tile_ox, R tile_oy, R px[4], R py[4]) {
    R cl[4][4];
    for (int k = 0; k < 4; ++k) mat4_mul_point(c->vp, v[k], cl[k]);
    int any_behind = (cl[0][3] <= 0) || (cl[1][3] <= 0) || (cl[2][3] <= 0) || (cl[3][3] <= 0);
    R W = (R)c->W, H = (R)c->H;
    for (int k = 0; k < 4; ++k) {
        px[k] = 0; py[k] = 0;
        if (!any_behind) {
            px[k] = (cl[k][0] / cl[k][3] + (R)1) * (R)0.5 * W - tile_ox;
            py[k] = ((R)1 - cl[k][1] / cl[k][3]) * (R)0.5 * H - tile_oy;
        }
    }
    return any_behind;
}

/* Row span for tile-local row `row` (rasterize_compute.wgsl:170-243 when
 * vertex_rows, backward_tiled_compute.wgsl:242-283 otherwise).  Returns 1 and
 * fills [xl_i, xr_i] if the row has a non-empty clamped span. */
static int row_span(int any_behind, const R px[4], const R py[4], uint32_t row, int TS, int vertex_rows,
                    int32_t* xl_o, int32_t* xr_o) {
    R xl = (R)1e10, xr = (R)-1e10;
    if (!any_behind) {
        R yc = (R)row + (R)0.5;
        for (int e = 0; e < 6; ++e) {
            R yi = py[EI[e]], yj = py[EJ[e]];
            if ((yi <= yc && yj > yc) || (yj <= yc && yi > yc)) {
                R t = (yc - yi) / (yj - yi);
                R x = px[EI[e]] + t * (px[EJ[e]] - px[EI[e]]);
                xl = RMIN(xl, x);
                xr = RMAX(xr, x);
            }
        }
        if (vertex_rows) {
            for (int k = 0; k < 4; ++k) {
                R vy = py[k];
                if (vy >= yc - (R)0.5 && vy < yc + (R)0.5) {
                    xl = RMIN(xl, px[k]);
                    xr = RMAX(xr, px[k]);
                }
            }
        }
    }
    if (!(xl <= xr)) return 0;
    R eps = (R)0.001;
    int32_t a = f2i(RCEIL(xl - (R)0.5 - eps));
    if (a < 0) a = 0;
    int32_t b = f2i(RFLOOR(xr - (R)0.5 + eps));
    if (b > TS - 1) b = TS - 1;
    if (a > b) return 0;
    *xl_o = a;
    *xr_o = b;
    return 1;
}

static void face_normals(const V3 v[4], V3 n[4]) {
    for (int f = 0; f < 4; ++f) {
        V3 va = v[FACES[f][0]], vb = v[FACES[f][1]], vc = v[FACES[f][2]];
        V3 nn = vcross(vsub(vc, va), vsub(vb, va));
        if (vdot(nn, vsub(v[FACES[f][3]], va)) < (R)0) nn = vneg(nn);
        n[f] = nn;
    }
}

/* Ray vs 4 inward planes: returns valid && t_min < t_max.  Tracks the entry
 * face (forward, strict >) and exit face (backward, strict <). */
static int intersect(const V3 v[4], const V3 n[4], V3 o, V3 d, R* tmin, R* tmax, int* entry, int* exitf) {
    R t_min = (R)-3.402823e38, t_max = (R)3.402823e38;
    int e_idx = 4, min_face = 0, max_face = 0, valid = 1;
    for (int f = 0; f < 4; ++f) {
        V3 va = v[FACES[f][0]];
        R num = vdot(n[f], vsub(va, o));
        R den = vdot(n[f], d);
        if (RABS(den) < (R)1e-20) {
            if (num > (R)0) valid = 0;
            continue;
        }
        R t = num / den;
        if (den > (R)0) {
            if (t > t_min) { t_min = t; e_idx = f; min_face = f; }
        } else {
            if (t < t_max) { t_max = t; max_face = f; }
        }
    }
    *tmin = t_min; *tmax = t_max;
    if (entry) *entry = e_idx;
    if (exitf) { exitf[0] = min_face; exitf[1] = max_face; }
    return valid && t_min < t_max;
}

/* ======================================================================== */
/* orc_rasterize -- rasterize_compute.wgsl:92-511.  rgba[H*W*4];           */
/* aux[H*W*8] (nullable); stats[H*W*4] (nullable).                         */
/* ======================================================================== */
EXPORT void SFX(orc_rasterize)(const R* verts, const uint32_t* idx, const R* colors, const R* dens,
                               const R* cgrad, const uint32_t* vals, const uint32_t* ranges, const R* vp,
                               const R* c2w, const R* intr, const R* cam3, int W, int H, int TS, R min_t,
                               R* rgba, R* aux, uint32_t* stats, const R* aux_data, int aux_dim) {
    Cam cm = {vp, c2w, intr, cam3, W, H, TS, min_t};
    uint32_t tiles_x = (uint32_t)((W + TS - 1) / TS), tiles_y = (uint32_t)((H + TS - 1) / TS);
    int64_t ntiles = (int64_t)tiles_x * tiles_y;
    V3 cam = v3(cam3[0], cam3[1], cam3[2]);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t tile = 0; tile < ntiles; ++tile) {
        uint32_t tile_x = (uint32_t)(tile % tiles_x), tile_y = (uint32_t)(tile / tiles_x);
        R tile_ox = (R)(tile_x * (uint32_t)TS), tile_oy = (R)(tile_y * (uint32_t)TS);
        int np = TS * TS;
        R col[256][4], nd[256][4], ent[256][4];
        R* cust = aux_dim > 0 ? (R*)calloc((size_t)256 * aux_dim, sizeof(R)) : NULL;  /* :458-462 */
        uint32_t st[256][4];
        memset(col, 0, sizeof(col)); memset(nd, 0, sizeof(nd)); memset(ent, 0, sizeof(ent)); memset(st, 0, sizeof(st));
        uint32_t rs = ranges[2 * tile], re = ranges[2 * tile + 1];
        uint32_t cursor = re;
        while (cursor > rs) {
            cursor -= 1u;
            uint32_t t = vals[cursor];
            V3 v[4];
            for (int k = 0; k < 4; ++k) v[k] = load_v3(verts, idx[4 * t + k]);
            R px4[4], py4[4];
            int any_behind = tile_proj(&cm, v, tile_ox, tile_oy, px4, py4);
            int32_t xl[16], xr[16];
            for (int r = 0; r < TS; ++r) {
                int32_t a, b;
                if (row_span(any_behind, px4, py4, (uint32_t)r, TS, 1, &a, &b)) {
                    /* trim saturated pixels from the row ends (:257-262) */
                    while (a <= b && col[r * TS + a][3] < (R)-13.8) a++;
                    while (b >= a && col[r * TS + b][3] < (R)-13.8) b--;
                    xl[r] = a; xr[r] = b;
                } else { xl[r] = 0; xr[r] = -1; }
            }
            R density = dens[t];
            V3 ctet = load_v3(colors, t), g = load_v3(cgrad, t);
            V3 n[4];
            face_normals(v, n);
            for (int r = 0; r < TS; ++r) {
                for (int32_t cc = xl[r]; cc <= xr[r]; ++cc) {
                    int pl = r * TS + cc;
                    uint32_t pxg = tile_x * (uint32_t)TS + (uint32_t)cc, pyg = tile_y * (uint32_t)TS + (uint32_t)r;
                    if (pxg >= (uint32_t)W || pyg >= (uint32_t)H) continue;
                    if (col[pl][3] < (R)-13.8) { st[pl][2]++; continue; }
                    V3 d = pixel_dir(&cm, pxg, pyg);
                    V3 o = vadd(cam, vscale(d, min_t));
                    R tmin, tmax;
                    int efi;
                    if (!intersect(v, n, o, d, &tmin, &tmax, &efi, NULL)) { st[pl][0]++; continue; }
                    R boff = vdot(g, vsub(o, v[0]));
                    V3 bc = vadd(ctet, v3(boff, boff, boff));
                    R dcdt = vdot(g, d);
                    V3 cs = vmax0(vadd(bc, v3(dcdt * tmin, dcdt * tmin, dcdt * tmin)));
                    V3 ce = vmax0(vadd(bc, v3(dcdt * tmax, dcdt * tmax, dcdt * tmax)));
                    R dist = tmax - tmin;
                    R od = clipr(density * dist, (R)1e-8, (R)88.0);
                    R alpha_t = safe_exp(-od);
                    R ph = phi(od);
                    R w0 = ph - alpha_t, w1 = (R)1 - ph;
                    V3 cp = vclip(vadd(vscale(ce, w0), vscale(cs, w1)), (R)0, MAX_VAL);
                    R alpha = (R)1 - alpha_t;
                    R Tj = safe_exp(col[pl][3]);
                    if (od < (R)0.01) st[pl][1]++;
                    else if (Tj < (R)1e-6) st[pl][2]++;
                    else st[pl][3]++;
                    if (Tj >= (R)1e-6) {
                        col[pl][0] += cp.x * Tj; col[pl][1] += cp.y * Tj; col[pl][2] += cp.z * Tj;
                        col[pl][3] = col[pl][3] - od;
                        V3 en = v3(0, 0, 0);
                        if (efi < 4) en = vnormalize(vneg(n[efi]));
                        R dp = w0 * tmax + w1 * tmin;
                        R ta = Tj * alpha;
                        nd[pl][0] += ta * en.x; nd[pl][1] += ta * en.y; nd[pl][2] += ta * en.z;
                        nd[pl][3] += Tj * dp;
                        R wt = alpha * Tj;
                        R cmid = (tmin + tmax) * (R)0.5;
                        R wc = wt * cmid;
                        ent[pl][0] += wt;
                        ent[pl][1] += wt > (R)1e-20 ? wt * RLOG(wt) : (R)0;
                        ent[pl][2] += wt * cmid;
                        ent[pl][3] += wc > (R)1e-20 ? wc * RLOG(wc) : (R)0;
                        for (int ai = 0; ai < aux_dim; ++ai) cust[pl * aux_dim + ai] += ta * aux_data[(size_t)t * aux_dim + ai];
                    }
                }
            }
        }
        for (int i = 0; i < np; ++i) {
            uint32_t rr = (uint32_t)i / (uint32_t)TS, cc = (uint32_t)i % (uint32_t)TS;
            uint32_t pxg = tile_x * (uint32_t)TS + cc, pyg = tile_y * (uint32_t)TS + rr;
            if (pxg >= (uint32_t)W || pyg >= (uint32_t)H) continue;
            size_t p = (size_t)pyg * (size_t)W + pxg;
            rgba[4 * p + 0] = col[i][0]; rgba[4 * p + 1] = col[i][1]; rgba[4 * p + 2] = col[i][2];
            rgba[4 * p + 3] = (R)1 - safe_exp(col[i][3]);
            if (aux) {
                size_t st_ = (size_t)(8 + aux_dim);
                for (int k = 0; k < 4; ++k) { aux[st_ * p + k] = nd[i][k]; aux[st_ * p + 4 + k] = ent[i][k]; }
                for (int ai = 0; ai < aux_dim; ++ai) aux[st_ * p + 8 + ai] = cust[i * aux_dim + ai];
            }
            if (stats) for (int k = 0; k < 4; ++k) stats[4 * p + k] = st[i][k];
        }
        free(cust);
    }
}

/* ======================================================================== */
/* orc_error_stats -- crates/rmesh-error/src/wgsl/error_tiled_compute.wgsl:  */
/* 90-373: the forward's front-to-back tile walk (vertex-row spans, no end   */
/* trimming), skipping pixels whose log transmittance fell below -5.5; each  */
/* covered pixel with T >= 1e-6 adds, with w = T * od, to its tet:           */
/* tet_err[16t + 0] w, [1] w pe, [2] w pe^2, [5] w se, [6..8] w entry,       */
/* [9..11] w exit, [12] w, [13..15] w centroid; tet_count[2t] += 1,          */
/* tet_count[2t+1] = max(., i32(65535 w)).  Serial, accumulated in double.   */
/* ======================================================================== */
EXPORT void SFX(orc_error_stats)(const R* verts, const uint32_t* idx, const R* dens, const uint32_t* vals,
                                 const uint32_t* ranges, const R* vp, const R* c2w, const R* intr, const R* cam3,
                                 int W, int H, int TS, R min_t, const R* pixel_err, const R* ssim_err,
                                 double* tet_err, int32_t* tet_count) {
    Cam cm = {vp, c2w, intr, cam3, W, H, TS, min_t};
    uint32_t tiles_x = (uint32_t)((W + TS - 1) / TS), tiles_y = (uint32_t)((H + TS - 1) / TS);
    int64_t ntiles = (int64_t)tiles_x * tiles_y;
    V3 cam = v3(cam3[0], cam3[1], cam3[2]);
    for (int64_t tile = 0; tile < ntiles; ++tile) {
        uint32_t tile_x = (uint32_t)(tile % tiles_x), tile_y = (uint32_t)(tile / tiles_x);
        R tile_ox = (R)(tile_x * (uint32_t)TS), tile_oy = (R)(tile_y * (uint32_t)TS);
        R logt[256];
        for (int i = 0; i < 256; ++i) logt[i] = 0;
        uint32_t rs = ranges[2 * tile], re = ranges[2 * tile + 1];
        uint32_t cursor = re;
        while (cursor > rs) {
            cursor -= 1u;
            uint32_t t = vals[cursor];
            V3 v[4];
            for (int k = 0; k < 4; ++k) v[k] = load_v3(verts, idx[4 * t + k]);
            R px4[4], py4[4];
            int any_behind = tile_proj(&cm, v, tile_ox, tile_oy, px4, py4);
            V3 n[4];
            face_normals(v, n);
            V3 cen = vscale(vadd(vadd(vadd(v[0], v[1]), v[2]), v[3]), (R)0.25);
            for (int r = 0; r < TS; ++r) {
                int32_t xa, xb;
                if (!row_span(any_behind, px4, py4, (uint32_t)r, TS, 1, &xa, &xb)) continue;
                for (int32_t cc = xa; cc <= xb; ++cc) {
                    int pl = r * TS + cc;
                    uint32_t pxg = tile_x * (uint32_t)TS + (uint32_t)cc, pyg = tile_y * (uint32_t)TS + (uint32_t)r;
                    if (pxg >= (uint32_t)W || pyg >= (uint32_t)H) continue;
                    if (logt[pl] < (R)-5.5) continue;
                    V3 d = pixel_dir(&cm, pxg, pyg);
                    V3 o = vadd(cam, vscale(d, min_t));
                    R tmin, tmax;
                    int efi;
                    if (!intersect(v, n, o, d, &tmin, &tmax, &efi, NULL)) continue;
                    R od = clipr(dens[t] * (tmax - tmin), (R)1e-8, (R)88.0);
                    R trans = safe_exp(logt[pl]);
                    if (trans < (R)1e-6) continue;
                    R w = trans * od;
                    V3 en = vadd(o, vscale(d, tmin)), ex = vadd(o, vscale(d, tmax));
                    size_t pidx = (size_t)pyg * (size_t)W + pxg;
                    double pe = (double)pixel_err[pidx], se = (double)ssim_err[pidx], wd = (double)w;
                    double* e = tet_err + 16 * (size_t)t;
                    e[0] += wd; e[1] += wd * pe; e[2] += wd * pe * pe; e[5] += wd * se;
                    e[6] += wd * en.x; e[7] += wd * en.y; e[8] += wd * en.z;
                    e[9] += wd * ex.x; e[10] += wd * ex.y; e[11] += wd * ex.z;
                    e[12] += wd; e[13] += wd * cen.x; e[14] += wd * cen.y; e[15] += wd * cen.z;
                    tet_count[2 * t] += 1;
                    int32_t q = f2i((R)65535 * w);
                    if (q > tet_count[2 * t + 1]) tet_count[2 * t + 1] = q;
                    logt[pl] -= od;
                }
            }
        }
    }
}

/* ======================================================================== */
/* orc_loss -- loss_compute.wgsl:24-72 plus the host loss value the         */
/* reference tests compute (kernel_tests.rs:869-878): sum over pixels and   */
/* RGB of (r-gt)^2 / n_pixels (L2) or |r-gt| / n_pixels (L1), in double.   */
/* ======================================================================== */
EXPORT double SFX(orc_loss)(int W, int H, int loss_type, const R* rendered, const R* gt, R* dl) {
    R npix = (R)((uint32_t)W * (uint32_t)H);
    double acc = 0.0;
    for (int64_t p = 0; p < (int64_t)W * H; ++p) {
        for (int c = 0; c < 3; ++c) {
            R diff = rendered[4 * p + c] - gt[3 * p + c];
            R g;
            if (loss_type == 0) g = (diff > 0 ? (R)1 : (diff < 0 ? (R)-1 : (R)0)) / npix;
            else g = (R)2 * diff / npix;
            if (dl) dl[4 * p + c] = g;
            double dd = (double)rendered[4 * p + c] - (double)gt[3 * p + c];
            acc += loss_type == 0 ? fabs(dd) : dd * dd;
        }
        if (dl) dl[4 * p + 3] = (R)0;
    }
    return acc / (double)W / (double)H;
}

/* ======================================================================== */
/* orc_backward -- backward_tiled_compute.wgsl:154-587.  Gradients are      */
/* accumulated (+=) into d_verts[3N], d_dens[M], d_cgrad[3M], d_base[3M].  */
/* threads <= 1 runs tiles in order (deterministic sums).                  */
/* ======================================================================== */
/* Custom aux channels (aux_dim > 0, dl_aux != NULL): the forward composites   */
/* aux[p][ai] += T alpha a[t][ai] (rasterize_compute.wgsl:458-462), i.e. each  */
/* item adds the "colour" alpha a[t] with weight T.  Its adjoint follows the    */
/* colour chain of this kernel: with s = sum_ai dl_aux[p][ai] a[t][ai], the     */
/* running d(log T) gains alpha s T_prev, the item's optical depth gains        */
/* T_prev alpha_t s (d alpha / d od = alpha_t), and d_aux[t][ai] gains          */
/* dl_aux[p][ai] T_prev alpha.  (The reference's only aux adjoint is in its     */
/* interval-tiled render mode, backward_interval_tiled.wgsl:637-649, whose d_aux */
/* term is the same and whose optical-depth term is an approximation; the tiled */
/* path has none.)                                                              */
static void backward_tile(const Cam* cm, int64_t tile, const R* verts, const uint32_t* idx, const R* colors,
                          const R* dens, const R* cgrad, const uint32_t* vals, const uint32_t* ranges,
                          const R* dl, const R* rendered, R* d_verts, R* d_dens, R* d_cgrad, R* d_base,
                          int use_atomics, const R* aux_data, int aux_dim, const R* dl_aux, R* d_aux) {
    if (!dl_aux || !aux_data) aux_dim = 0;
    R acc_aux[64];
    int W = cm->W, H = cm->H, TS = cm->TS;
    uint32_t tiles_x = (uint32_t)((W + TS - 1) / TS);
    uint32_t tile_x = (uint32_t)(tile % tiles_x), tile_y = (uint32_t)(tile / tiles_x);
    R tile_ox = (R)(tile_x * (uint32_t)TS), tile_oy = (R)(tile_y * (uint32_t)TS);
    V3 cam = v3(cm->cam[0], cm->cam[1], cm->cam[2]);
    R st[256][4], dlt[256];
    for (int i = 0; i < TS * TS; ++i) {
        uint32_t rr = (uint32_t)i / (uint32_t)TS, cc = (uint32_t)i % (uint32_t)TS;
        uint32_t pxg = tile_x * (uint32_t)TS + cc, pyg = tile_y * (uint32_t)TS + rr;
        if (pxg < (uint32_t)W && pyg < (uint32_t)H) {
            size_t p = (size_t)pyg * (size_t)W + pxg;
            R a = rendered[4 * p + 3];
            st[i][0] = rendered[4 * p]; st[i][1] = rendered[4 * p + 1]; st[i][2] = rendered[4 * p + 2];
            st[i][3] = RLOG(RMAX((R)1 - a, (R)1e-20));
            dlt[i] = -dl[4 * p + 3] * ((R)1 - a);
        } else {
            st[i][0] = st[i][1] = st[i][2] = st[i][3] = 0; dlt[i] = 0;
        }
    }
    uint32_t rs = ranges[2 * tile], re = ranges[2 * tile + 1];
    for (uint32_t cursor = rs; cursor < re; ++cursor) {
        uint32_t t = vals[cursor];
        V3 v[4];
        uint32_t vi[4];
        for (int k = 0; k < 4; ++k) { vi[k] = idx[4 * t + k]; v[k] = load_v3(verts, vi[k]); }
        R px4[4], py4[4];
        int any_behind = tile_proj(cm, v, tile_ox, tile_oy, px4, py4);
        int32_t xl[16], xr[16];
        for (int r = 0; r < TS; ++r)
            if (!row_span(any_behind, px4, py4, (uint32_t)r, TS, 0, &xl[r], &xr[r])) { xl[r] = 0; xr[r] = -1; }
        R density = dens[t];
        V3 ctet = load_v3(colors, t), g = load_v3(cgrad, t);
        V3 n[4];
        face_normals(v, n);
        R acc_d = 0;
        for (int ai = 0; ai < aux_dim; ++ai) acc_aux[ai] = 0;
        V3 acc_v[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        V3 acc_g = {0, 0, 0}, acc_b = {0, 0, 0};
        for (int r = 0; r < TS; ++r) {
            for (int32_t cc = xl[r]; cc <= xr[r]; ++cc) {
                int pl = r * TS + cc;
                uint32_t pxg = tile_x * (uint32_t)TS + (uint32_t)cc, pyg = tile_y * (uint32_t)TS + (uint32_t)r;
                if (pxg >= (uint32_t)W || pyg >= (uint32_t)H) continue;
                size_t p = (size_t)pyg * (size_t)W + pxg;
                V3 d = pixel_dir(cm, pxg, pyg);
                R tmin, tmax;
                int mf[2];
                if (!intersect(v, n, cam, d, &tmin, &tmax, NULL, mf)) continue;
                R boff = vdot(g, vsub(cam, v[0]));
                V3 bc = vadd(ctet, v3(boff, boff, boff));
                R dcdt = vdot(g, d);
                V3 csr = vadd(bc, v3(dcdt * tmin, dcdt * tmin, dcdt * tmin));
                V3 cer = vadd(bc, v3(dcdt * tmax, dcdt * tmax, dcdt * tmax));
                V3 cs = vmax0(csr), ce = vmax0(cer);
                R dist = tmax - tmin;
                R od = clipr(density * dist, (R)1e-8, (R)88.0);
                R alpha_t = safe_exp(-od);
                R ph = phi(od);
                R w0 = ph - alpha_t, w1 = (R)1 - ph;
                V3 cp = vclip(vadd(vscale(ce, w0), vscale(cs, w1)), MIN_VAL, MAX_VAL);
                V3 color = v3(st[pl][0], st[pl][1], st[pl][2]);
                R log_t = st[pl][3];
                R d_log_t = dlt[pl];
                R prev_log_t = RMIN(log_t + od, (R)0);
                R t_prev = safe_exp(prev_log_t);
                V3 prev_color = vsub(color, vscale(cp, t_prev));
                st[pl][0] = prev_color.x; st[pl][1] = prev_color.y; st[pl][2] = prev_color.z; st[pl][3] = prev_log_t;
                if (t_prev < (R)1e-6) { dlt[pl] = d_log_t; continue; }
                V3 dcol = v3(dl[4 * p], dl[4 * p + 1], dl[4 * p + 2]);
                V3 dcp = vclip(vscale(dcol, t_prev), MIN_VAL, MAX_VAL);
                R d_od_state = -d_log_t;
                R aux_s = 0;  /* sum_ai dl_aux[p][ai] a[t][ai] */
                for (int ai = 0; ai < aux_dim; ++ai)
                    aux_s += dl_aux[(size_t)p * aux_dim + ai] * aux_data[(size_t)t * aux_dim + ai];
                R alpha = (R)1 - alpha_t;
                R d_old = clipr(d_log_t + (vdot(dcol, cp) + alpha * aux_s) * t_prev, MIN_VAL, MAX_VAL);
                dlt[pl] = d_old;
                R dph = dphi_dx(od);
                R dw0 = dph + alpha_t, dw1 = -dph;
                V3 dce_i = vscale(dcp, w0), dcs_i = vscale(dcp, w1);
                R d_od_int = vdot(dcp, vadd(vscale(ce, dw0), vscale(cs, dw1))) + t_prev * alpha_t * aux_s;
                for (int ai = 0; ai < aux_dim; ++ai) acc_aux[ai] += dl_aux[(size_t)p * aux_dim + ai] * t_prev * alpha;
                R d_od = clipr(d_od_state + d_od_int, MIN_VAL, MAX_VAL);
                R od_raw = density * dist;
                int active = (od_raw >= (R)1e-8) && (od_raw <= (R)88.0);
                R d_od_raw = active ? d_od : (R)0;
                R d_dens_l = clipr(d_od_raw * dist, MIN_VAL, MAX_VAL);
                R d_dist = clipr(d_od_raw * density, MIN_VAL, MAX_VAL);
                R d_tmin = -d_dist, d_tmax = d_dist;
                V3 dcsr = v3(csr.x > 0 ? dcs_i.x : 0, csr.y > 0 ? dcs_i.y : 0, csr.z > 0 ? dcs_i.z : 0);
                V3 dcer = v3(cer.x > 0 ? dce_i.x : 0, cer.y > 0 ? dce_i.y : 0, cer.z > 0 ? dce_i.z : 0);
                V3 dbase = vadd(dcsr, dcer);
                R ss = (dcsr.x + dcsr.y) + dcsr.z, se = (dcer.x + dcer.y) + dcer.z;
                R d_dcdt = ss * tmin + se * tmax;
                d_tmin += ss * dcdt;
                d_tmax += se * dcdt;
                R sb = (dbase.x + dbase.y) + dbase.z;
                V3 dgl = vscale(vsub(cam, v[0]), sb);
                V3 dv0b = vscale(vneg(g), sb);
                dgl = vadd(dgl, vscale(d, d_dcdt));
                acc_b = vadd(acc_b, vclip(dbase, MIN_VAL, MAX_VAL));
                V3 dvl[4] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                for (int s = 0; s < 2; ++s) {
                    int f = mf[s];
                    R dt = s == 0 ? d_tmin : d_tmax;
                    R tt = s == 0 ? tmin : tmax;
                    V3 va = v[FACES[f][0]], vb = v[FACES[f][1]], vc = v[FACES[f][2]];
                    V3 nn = vcross(vsub(vc, va), vsub(vb, va));
                    R den = vdot(nn, d);
                    R inv_den = safe_div((R)1, den);
                    V3 hit = vadd(cam, vscale(d, tt));
                    V3 dta = vscale(vadd(vcross(vsub(va, hit), vsub(vb, vc)), nn), inv_den);
                    V3 dtb = vscale(vcross(vsub(va, hit), vsub(vc, va)), inv_den);
                    V3 dtc = vscale(vcross(vsub(va, hit), vsub(va, vb)), inv_den);
                    dvl[FACES[f][0]] = vadd(dvl[FACES[f][0]], vclip(vscale(dta, dt), MIN_VAL, MAX_VAL));
                    dvl[FACES[f][1]] = vadd(dvl[FACES[f][1]], vclip(vscale(dtb, dt), MIN_VAL, MAX_VAL));
                    dvl[FACES[f][2]] = vadd(dvl[FACES[f][2]], vclip(vscale(dtc, dt), MIN_VAL, MAX_VAL));
                }
                dvl[0] = vadd(dvl[0], dv0b);
                acc_d += clipr(d_dens_l, MIN_VAL, MAX_VAL);
                for (int k = 0; k < 4; ++k) acc_v[k] = vadd(acc_v[k], vclip(dvl[k], MIN_VAL, MAX_VAL));
                acc_g = vadd(acc_g, vclip(dgl, MIN_VAL, MAX_VAL));
            }
        }
        for (int ai = 0; ai < aux_dim; ++ai) {
            if (use_atomics) {
#pragma omp atomic
                d_aux[(size_t)t * aux_dim + ai] += acc_aux[ai];
            } else {
                d_aux[(size_t)t * aux_dim + ai] += acc_aux[ai];
            }
        }
        if (use_atomics) {
#pragma omp atomic
            d_dens[t] += acc_d;
            for (int k = 0; k < 4; ++k) {
#pragma omp atomic
                d_verts[3 * vi[k] + 0] += acc_v[k].x;
#pragma omp atomic
                d_verts[3 * vi[k] + 1] += acc_v[k].y;
#pragma omp atomic
                d_verts[3 * vi[k] + 2] += acc_v[k].z;
            }
#pragma omp atomic
            d_cgrad[3 * t + 0] += acc_g.x;
#pragma omp atomic
            d_cgrad[3 * t + 1] += acc_g.y;
#pragma omp atomic
            d_cgrad[3 * t + 2] += acc_g.z;
#pragma omp atomic
            d_base[3 * t + 0] += acc_b.x;
#pragma omp atomic
            d_base[3 * t + 1] += acc_b.y;
#pragma omp atomic
            d_base[3 * t + 2] += acc_b.z;
        } else {
            d_dens[t] += acc_d;
            for (int k = 0; k < 4; ++k) {
                d_verts[3 * vi[k] + 0] += acc_v[k].x;
                d_verts[3 * vi[k] + 1] += acc_v[k].y;
                d_verts[3 * vi[k] + 2] += acc_v[k].z;
            }
            d_cgrad[3 * t + 0] += acc_g.x; d_cgrad[3 * t + 1] += acc_g.y; d_cgrad[3 * t + 2] += acc_g.z;
            d_base[3 * t + 0] += acc_b.x; d_base[3 * t + 1] += acc_b.y; d_base[3 * t + 2] += acc_b.z;
        }
    }
}

/* orc_backward_aux -- orc_backward plus the custom aux channels' adjoint     */
/* (see backward_tile): aux_data [M][aux_dim], dl_aux [H*W][aux_dim]; d_aux   */
/* [M][aux_dim] is accumulated (+=).  aux_dim <= 64.                          */
EXPORT void SFX(orc_backward_aux)(const R* verts, const uint32_t* idx, const R* colors, const R* dens,
                                  const R* cgrad, const uint32_t* vals, const uint32_t* ranges, const R* vp,
                                  const R* c2w, const R* intr, const R* cam3, int W, int H, int TS, const R* dl,
                                  const R* rendered, R* d_verts, R* d_dens, R* d_cgrad, R* d_base, int threads,
                                  const R* aux_data, int aux_dim, const R* dl_aux, R* d_aux) {
    Cam cm = {vp, c2w, intr, cam3, W, H, TS, (R)0};
    uint32_t tiles_x = (uint32_t)((W + TS - 1) / TS), tiles_y = (uint32_t)((H + TS - 1) / TS);
    int64_t ntiles = (int64_t)tiles_x * tiles_y;
    if (aux_dim > 64) aux_dim = 64;
    if (threads <= 1) {
        for (int64_t tile = 0; tile < ntiles; ++tile)
            backward_tile(&cm, tile, verts, idx, colors, dens, cgrad, vals, ranges, dl, rendered, d_verts, d_dens,
                          d_cgrad, d_base, 0, aux_data, aux_dim, dl_aux, d_aux);
    } else {
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
        for (int64_t tile = 0; tile < ntiles; ++tile)
            backward_tile(&cm, tile, verts, idx, colors, dens, cgrad, vals, ranges, dl, rendered, d_verts, d_dens,
                          d_cgrad, d_base, 1, aux_data, aux_dim, dl_aux, d_aux);
    }
}

EXPORT void SFX(orc_backward)(const R* verts, const uint32_t* idx, const R* colors, const R* dens, const R* cgrad,
                              const uint32_t* vals, const uint32_t* ranges, const R* vp, const R* c2w,
                              const R* intr, const R* cam3, int W, int H, int TS, const R* dl, const R* rendered,
                              R* d_verts, R* d_dens, R* d_cgrad, R* d_base, int threads) {
    SFX(orc_backward_aux)(verts, idx, colors, dens, cgrad, vals, ranges, vp, c2w, intr, cam3, W, H, TS, dl, rendered,
                          d_verts, d_dens, d_cgrad, d_base, threads, NULL, 0, NULL, NULL);
}

/* ======================================================================== */
/* orc_sh_backward -- adjoint of the SH colour (project_compute.wgsl:264-318) */
/* which the reference does not have.  For each tet with visible[t], chains  */
/* d_colors (the adjoint's colour gradient) through softplus, the SH basis,   */
/* the colour-gradient offset dot(g, v0 - centroid) and the view direction   */
/* normalize(centroid - cam): writes d_sh [M][3][nc] and ADDS to d_verts     */
/* [3N] and d_cgrad [3M].  Serial (deterministic vertex sums).               */
/* ======================================================================== */
EXPORT void SFX(orc_sh_backward)(int64_t M, const R* verts, const uint32_t* idx, const R* cgrad, const R* sh,
                                 int sh_degree, const R* cam3, const uint8_t* visible, const R* d_colors,
                                 R* d_sh, R* d_verts, R* d_cgrad) {
    uint32_t nc = (uint32_t)((sh_degree + 1) * (sh_degree + 1));
    memset(d_sh, 0, sizeof(R) * (size_t)M * 3u * nc);
    for (int64_t t = 0; t < M; ++t) {
        if (!visible[t]) continue;
        R dc[3] = {d_colors[3 * t], d_colors[3 * t + 1], d_colors[3 * t + 2]};
        if (dc[0] == (R)0 && dc[1] == (R)0 && dc[2] == (R)0) continue;
        V3 v[4];
        for (int k = 0; k < 4; ++k) v[k] = load_v3(verts, idx[4 * t + k]);
        V3 centroid, dir;
        R len = sh_dir(v, cam3, &centroid, &dir);
        const R* co = sh + (size_t)t * 3u * nc;
        R* dco = d_sh + (size_t)t * 3u * nc;
        V3 g = load_v3(cgrad, t);
        V3 v0c = vsub(v[0], centroid);
        R off = vdot(g, v0c);
        R sum_drgb = 0;
        V3 d_dir = v3(0, 0, 0);
        for (uint32_t c = 0; c < 3; ++c) {
            R val = 0;
            for (uint32_t i = 0; i < nc; ++i) val += sh_basis(i, dir.x, dir.y, dir.z) * co[c * nc + i];
            R drgb = dc[c] * dsoftplus(val + (R)0.5 + off);
            sum_drgb += drgb;
            for (uint32_t i = 0; i < nc; ++i) {
                dco[c * nc + i] = drgb * sh_basis(i, dir.x, dir.y, dir.z);
                d_dir = vadd(d_dir, vscale(sh_basis_grad(i, dir.x, dir.y, dir.z), drgb * co[c * nc + i]));
            }
        }
        /* offset = dot(g, v0 - centroid) */
        d_cgrad[3 * t] += sum_drgb * v0c.x;
        d_cgrad[3 * t + 1] += sum_drgb * v0c.y;
        d_cgrad[3 * t + 2] += sum_drgb * v0c.z;
        V3 d_centroid = vscale(g, -sum_drgb);
        V3 d_v0 = vscale(g, sum_drgb);
        /* dir = raw / |raw|, raw = centroid - cam */
        if (len > (R)0) {
            R dd = vdot(dir, d_dir);
            d_centroid = vadd(d_centroid, vscale(vsub(d_dir, vscale(dir, dd)), (R)1 / len));
        }
        for (int k = 0; k < 4; ++k) {
            uint32_t vi = idx[4 * t + k];
            V3 dv = vscale(d_centroid, (R)0.25);
            if (k == 0) dv = vadd(dv, d_v0);
            d_verts[3 * vi] += dv.x;
            d_verts[3 * vi + 1] += dv.y;
            d_verts[3 * vi + 2] += dv.z;
        }
    }
}

/* ======================================================================== */
/* orc_adam -- adam_compute.wgsl:121-149 for one parameter group.          */
/* ======================================================================== */
EXPORT void SFX(orc_adam)(int64_t n, R* params, const R* grads, R* m, R* v, uint32_t step, R lr, R beta1, R beta2,
                          R eps) {
    R step_f = (R)step;
    for (int64_t i = 0; i < n; ++i) {
        R gr = grads[i];
        R g = clipr(gr != gr ? (R)0 : gr, MIN_VAL, MAX_VAL);
        R m_new = beta1 * m[i] + ((R)1 - beta1) * g;
        m[i] = m_new;
        R v_new = beta2 * v[i] + ((R)1 - beta2) * g * g;
        v[i] = v_new;
        R b1p = REXP(step_f * RLOG(beta1));
        R b2p = REXP(step_f * RLOG(beta2));
        R m_hat = safe_div(m_new, (R)1 - b1p);
        R v_hat = safe_div(v_new, (R)1 - b2p);
        params[i] -= lr * safe_div(m_hat, safe_sqrt(v_hat) + eps);
    }
}

/* ======================================================================== */
/* .rmesh scene file (crates/rmesh-data/src/lib.rs:142-393), on the        */
/* decompressed bytes.  Layout: u32 N, M, sh_degree, k; f32 pose[8];       */
/* f32 vertices[3N]; u32 indices[4M]; u8 log-densities[M]; align 4;        */
/* f16 SH mean[D], basis[k'][D], weights[M][k'] (D = 3 (deg+1)^2,          */
/* k' = min(k, D)); align 4; f16 colour gradients[3M] (zeros when a tagged */
/* "RMTX" section starts there, zero-padded when the file is short).       */
/* ======================================================================== */
static float half_bits_to_float(uint16_t h) {
    uint32_t sgn = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1Fu, m = h & 0x3FFu, bits;
    if (e == 0) {
        if (m == 0) {
            bits = sgn;
        } else { /* subnormal: renormalise */
            int ee = 127 - 15 + 1;
            while (!(m & 0x400u)) { m <<= 1; ee--; }
            bits = sgn | ((uint32_t)ee << 23) | ((m & 0x3FFu) << 13);
        }
    } else if (e == 31) {
        bits = sgn | 0x7F800000u | (m << 13);
    } else {
        bits = sgn | ((e - 15 + 127) << 23) | (m << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static uint32_t rd_u32(const uint8_t* d, int64_t off) { uint32_t v; memcpy(&v, d + off, 4); return v; }
static uint16_t rd_u16(const uint8_t* d, int64_t off) { uint16_t v; memcpy(&v, d + off, 2); return v; }

/* header -> hdr[0..3] = N, M, sh_degree, k; returns -1 when too short */
EXPORT int SFX(orc_rmesh_header)(const uint8_t* d, int64_t len, uint32_t* hdr) {
    if (len < 48) return -1;
    for (int i = 0; i < 4; ++i) hdr[i] = rd_u32(d, 4 * i);
    return 0;
}

/* Circumsphere of one tet in double precision with the loader's degenerate
 * handling (lib.rs:601-707). */
typedef struct { double x, y, z; } D3;
static D3 d3(double x, double y, double z) { D3 r = {x, y, z}; return r; }
static D3 d3sub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
static D3 d3add(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
static D3 d3scale(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
static double d3dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static D3 d3cross(D3 a, D3 b) { return d3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
static double d3len(D3 a) { return sqrt(d3dot(a, a)); }

static void circumsphere_f64(const float* verts, const uint32_t* q, float* out) {
    D3 v[4];
    for (int k = 0; k < 4; ++k)
        v[k] = d3((double)verts[3 * q[k]], (double)verts[3 * q[k] + 1], (double)verts[3 * q[k] + 2]);
    D3 a = d3sub(v[1], v[0]), b = d3sub(v[2], v[0]), c = d3sub(v[3], v[0]);
    double aa = d3dot(a, a), bb = d3dot(b, b), cc = d3dot(c, c);
    D3 bc = d3cross(b, c), ca = d3cross(c, a), ab = d3cross(a, b);
    double denom = 2.0 * d3dot(a, bc);
    if (fabs(denom) < 1e-10) {
        double md = d3len(d3sub(v[1], v[0]));
        md = fmax(md, d3len(d3sub(v[2], v[0])));
        md = fmax(md, d3len(d3sub(v[3], v[0])));
        md = fmax(md, d3len(d3sub(v[2], v[1])));
        md = fmax(md, d3len(d3sub(v[3], v[1])));
        md = fmax(md, d3len(d3sub(v[3], v[2])));
        D3 cen = d3scale(d3add(d3add(d3add(v[0], v[1]), v[2]), v[3]), 0.25);
        out[0] = (float)cen.x; out[1] = (float)cen.y; out[2] = (float)cen.z;
        if (md < 1e-7) {
            double r = d3len(d3sub(v[0], cen));
            r = fmin(r, d3len(d3sub(v[1], cen)));
            r = fmin(r, d3len(d3sub(v[2], cen)));
            r = fmin(r, d3len(d3sub(v[3], cen)));
            out[3] = (float)(r * r);
        } else {
            out[3] = 1e20f;
        }
        return;
    }
    D3 num = d3add(d3add(d3scale(bc, aa), d3scale(ca, bb)), d3scale(ab, cc));
    D3 rel = d3(num.x / denom, num.y / denom, num.z / denom);
    D3 cen = d3add(v[0], rel);
    out[0] = (float)cen.x; out[1] = (float)cen.y; out[2] = (float)cen.z;
    out[3] = (float)d3dot(rel, rel);
}

/* Decodes the whole file; arrays sized from the header.  Returns the byte
 * offset after the colour gradients, or -1 when the file is too short. */
EXPORT int64_t SFX(orc_rmesh_decode)(const uint8_t* d, int64_t len, float* pose7, float* verts, uint32_t* idx,
                                     float* dens, float* sh, float* grads, float* circ) {
    uint32_t N = rd_u32(d, 0), M = rd_u32(d, 4), deg = rd_u32(d, 8), k = rd_u32(d, 12);
    int64_t off = 16;
    for (int i = 0; i < 7; ++i) memcpy(&pose7[i], d + off + 4 * i, 4);
    off += 32;
    const uint32_t nc = (deg + 1u) * (deg + 1u), D = 3u * nc, K = k < D ? k : D;
    int64_t need = off + 12ll * N + 16ll * M + M;
    if (len < need) return -1;
    memcpy(verts, d + off, 12ull * N); off += 12ll * N;
    memcpy(idx, d + off, 16ull * M); off += 16ll * M;
    for (uint32_t t = 0; t < M; ++t) dens[t] = expf(((float)d[off + t] - 100.0f) / 20.0f);
    off += M;
    off = (off + 3) & ~(int64_t)3;
    if (len < off + 2ll * (D + (int64_t)K * D + (int64_t)M * K)) return -1;
    const int64_t mean_off = off, basis_off = off + 2ll * D, w_off = basis_off + 2ll * K * D;
    off = w_off + 2ll * M * K;
    for (uint32_t t = 0; t < M; ++t)
        for (uint32_t f = 0; f < D; ++f) {
            float val = half_bits_to_float(rd_u16(d, mean_off + 2ll * f));
            for (uint32_t q = 0; q < K; ++q)
                val += half_bits_to_float(rd_u16(d, w_off + 2ll * ((int64_t)t * K + q))) *
                       half_bits_to_float(rd_u16(d, basis_off + 2ll * ((int64_t)q * D + f)));
            sh[(int64_t)t * D + f] = val;
        }
    off = (off + 3) & ~(int64_t)3;
    const int64_t ng = 3ll * M;
    if (off + 4 <= len && rd_u32(d, off) == 0x524D5458u) {
        memset(grads, 0, sizeof(float) * ng);
    } else {
        int64_t avail = (len - off) / 2;
        if (avail > ng) avail = ng;
        for (int64_t i = 0; i < ng; ++i) grads[i] = i < avail ? half_bits_to_float(rd_u16(d, off + 2 * i)) : 0.0f;
        off += 2 * avail;
    }
    for (uint32_t t = 0; t < M; ++t) circumsphere_f64(verts, idx + 4ull * t, circ + 4ull * t);
    return off;
}

EXPORT void SFX(orc_set_threads)(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

EXPORT int SFX(orc_max_threads)(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
