/*
 * rmesh_b200.h -- C ABI of the B200-native rmeshvk tiled volume-rendering path.
 *
 * One context owns a tet mesh (fixed topology), its trainable parameters, the
 * Adam moments and every device buffer of the path.  Each entry point below
 * replaces one method of the reference's PyO3 class `RMeshRenderer`
 * (crates/rmesh-python/src/lib.rs); the comment on each names the method and
 * its lines.  Paths are relative to the reference repository root.
 *
 * Conventions
 *  - Every call returns an int status (RMESH_OK = 0).  rmesh_last_error()
 *    returns a message for the last failing call on that context.
 *  - Array pointers may be host memory or CUDA device memory (unified virtual
 *    addressing decides); device pointers avoid a host round trip.
 *  - Arrays are flat, C-contiguous, float32 / uint32, with the reference's
 *    layouts: vertices [3N], indices [4M], base_colors [3M], densities [M],
 *    color_grads [3M], circumdata [4M] = (cx, cy, cz, r^2), images [H][W][4]
 *    premultiplied RGBA, ground truth [H][W][3] RGB.
 *  - Work is ordered on the context's CUDA stream (rmesh_set_stream); calls
 *    that return host-visible results synchronise that stream.  A context is
 *    not thread-safe; use one per thread.
 */
#ifndef RMESH_B200_H
#define RMESH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RMESH_ABI_VERSION 2

#if defined(__GNUC__)
#define RMESH_API __attribute__((visibility("default")))
#else
#define RMESH_API
#endif

/* status codes */
#define RMESH_OK 0
#define RMESH_ERR_INVALID_ARG 1  /* bad sizes/pointers (reference: PyValueError) */
#define RMESH_ERR_CUDA 2         /* CUDA runtime error (reference: PyRuntimeError, lib.rs:306-329) */
#define RMESH_ERR_OOM 3          /* device allocation failed */
#define RMESH_ERR_PAIR_OVERFLOW 4 /* pair buffers too small even after growing to the limit */
#define RMESH_ERR_TIMEOUT 5      /* a bounded device spin gave up (kernel returned an error, no hang) */
#define RMESH_ERR_STATE 6        /* call order violated (e.g. backward before forward_tiled) */
#define RMESH_ERR_NO_DEVICE 7    /* no CUDA device / library built for another architecture */
#define RMESH_ERR_TOO_LARGE 8    /* input above the fixed scratch of rmesh_count_tiles_static */

typedef struct RmeshCtx RmeshCtx;

/* Mesh and initial parameters (reference constructor, lib.rs:265-277). */
typedef struct {
  int64_t n_vertices;        /* N */
  int64_t n_tets;            /* M */
  const float* vertices;     /* [3N] */
  const uint32_t* indices;   /* [4M] */
  const float* base_colors;  /* [3M] */
  const float* densities;    /* [M] */
  const float* color_grads;  /* [3M] */
  const float* circumdata;   /* [4M] */
  int32_t width;             /* default view size */
  int32_t height;
  int32_t aux_dim;           /* custom per-tet aux channels, 0..RMESH_MAX_AUX_DIM (lib.rs:264-266) */
  int32_t tile_size;         /* 0 -> 12, the reference's hard-coded value (lib.rs:442) */
  int32_t device;            /* CUDA device ordinal, -1 = current */
  int32_t sh_degree;         /* 0..3, used when sh_coeffs is set */
  const float* sh_coeffs;    /* NULL: colours are base_colors (the reference's training
                              * path, lib.rs:393-439); else [M][3][(sh_degree+1)^2]
                              * coefficients (coefficient c*nc + i of channel c), colour =
                              * softplus(SH(dir) + 0.5 + dot(g, v0 - centroid)) per view
                              * (project_compute.wgsl:264-318), read as f16 like the
                              * reference's packed buffer (rmesh-viewer/src/gpu_state.rs:60-88) */
  int32_t reserved[2];
} RmeshSceneDesc;

/* One view: the three arrays of the reference camera methods (lib.rs:1040-1048)
 * plus its image size. */
typedef struct {
  float cam_pos[3];
  float vp[16];              /* view-projection, column-major */
  float c2w_intrinsics[16];  /* c2w col0 xyz,0, col1 xyz,0, col2 xyz,0, fx,fy,cx,cy */
  int32_t width;
  int32_t height;
} RmeshCamera;

/* Options of the multi-view training step (no reference counterpart; the
 * learning rates and loss type are those of train_step, lib.rs:2405-2415). */
typedef struct {
  float lr_verts;
  float lr_dens;
  float lr_grads;
  float lr_base;      /* 0 keeps base colours fixed, as the reference train_step does */
  int32_t loss_type;  /* 0 = L1, 1 = L2 */
  int32_t mode;       /* RMESH_MODE_* */
  float lr_sh;        /* SH coefficients' learning rate (SH contexts; no reference counterpart) */
  int32_t reserved;
} RmeshTrainOpts;

#define RMESH_MODE_PLAIN 0    /* one launch sequence per view, one tile per CTA */
#define RMESH_MODE_BATCHED 1  /* all views in one launch sequence, persistent (view,tile) queue */
#define RMESH_MODE_GRAPH 2    /* BATCHED, captured as a CUDA graph per step signature (up to 8 kept) and replayed */

typedef struct {
  int64_t n_vertices, n_tets;
  int32_t width, height, tile_size, n_views_last;
  uint32_t step;
  uint32_t last_error_bits;      /* device status bits of the last run */
  uint64_t n_visible_last;       /* tile-touching (view, tet) pairs of the last run */
  uint64_t n_pairs_last;         /* (tile, tet) slots of the last run */
  uint64_t pair_capacity;
  uint64_t device_bytes;         /* device memory held by the context */
} RmeshInfo;

/* ---- lifetime ------------------------------------------------------------ */
/* RMeshRenderer.__new__ (lib.rs:265-870): copies every input to the device. */
RMESH_API int rmesh_create(const RmeshSceneDesc* desc, RmeshCtx** out);
RMESH_API int rmesh_destroy(RmeshCtx* ctx);
RMESH_API const char* rmesh_last_error(const RmeshCtx* ctx);
RMESH_API int rmesh_abi_version(void);

/* ---- settings ------------------------------------------------------------- */
RMESH_API int rmesh_set_stream(RmeshCtx* ctx, void* cuda_stream);     /* no reference counterpart */
RMESH_API int rmesh_set_min_t(RmeshCtx* ctx, float min_t);            /* set_min_t, lib.rs:873-875 */
RMESH_API int rmesh_set_tile_size(RmeshCtx* ctx, int32_t tile_size);  /* 8, 12 or 16 (reference fixes 12) */

/* ---- parameters ----------------------------------------------------------- */
/* update_params, lib.rs:2641-2669 (any pointer may be NULL to keep that group) */
RMESH_API int rmesh_update_params(RmeshCtx* ctx, const float* vertices, const float* base_colors,
                        const float* densities, const float* color_grads);
/* get_params, lib.rs:2674-2686 */
RMESH_API int rmesh_get_params(RmeshCtx* ctx, float* vertices, float* base_colors, float* densities,
                     float* color_grads);
/* getters step/width/height, lib.rs:2688-2705 */
RMESH_API int rmesh_get_info(RmeshCtx* ctx, RmeshInfo* info);

/* Optimiser state for checkpoints (no reference counterpart: the reference
 * keeps its Adam moments private).  The state is the first and second Adam
 * moments of every group back to back -- m and v of the vertices [3N], the
 * densities [M], the colour gradients [3M], the base colours [3M] and, in SH
 * contexts, the SH coefficients [3 nc M] -- plus the step count that drives
 * the bias correction.  rmesh_adam_state_size gives the length in floats;
 * state may be host or device memory.  With rmesh_get_params /
 * rmesh_update_params (and rmesh_get_sh / rmesh_update_sh) a run restored
 * from them continues as the saved one would. */
RMESH_API int rmesh_adam_state_size(RmeshCtx* ctx, uint64_t* n_floats);
RMESH_API int rmesh_get_adam_state(RmeshCtx* ctx, float* state, uint32_t* step);
RMESH_API int rmesh_set_adam_state(RmeshCtx* ctx, const float* state, uint32_t step);

/* set_aux_data / get_aux_data, lib.rs:892-921: the [M][aux_dim] custom
 * per-tet channels that forward_tiled's aux output composites after its eight
 * fixed channels (aux_out [H][W][8 + aux_dim]); zeros until set. */
#define RMESH_MAX_AUX_DIM 64
RMESH_API int rmesh_set_aux_data(RmeshCtx* ctx, const float* aux_data);
RMESH_API int rmesh_get_aux_data(RmeshCtx* ctx, float* aux_data);

/* SH coefficients of a context created with sh_coeffs (no reference
 * counterpart: the reference's binding trains base colours only).  get/update
 * copy [M][3][nc] floats; get_sh_grad returns the coefficient gradient of the
 * last rmesh_backward / training call; set_lr_sh sets the learning rate that
 * rmesh_train_step applies to them (default 0). */
RMESH_API int rmesh_update_sh(RmeshCtx* ctx, const float* sh_coeffs);
RMESH_API int rmesh_get_sh(RmeshCtx* ctx, float* sh_coeffs);
RMESH_API int rmesh_get_sh_grad(RmeshCtx* ctx, float* d_sh_coeffs);
RMESH_API int rmesh_set_lr_sh(RmeshCtx* ctx, float lr_sh);

/* ---- the path ------------------------------------------------------------- */
/* forward_tiled, lib.rs:1041-1204: project -> bin -> sort -> ranges -> composite.
 * rgba_out [H][W][4]; aux_out [H][W][8 + aux_dim] or NULL (render_aux). */
RMESH_API int rmesh_forward_tiled(RmeshCtx* ctx, const RmeshCamera* cam, float* rgba_out, float* aux_out);

/* Batched forward (no reference counterpart; the forward half of
 * rmesh_train_step_views): n_views cameras of any sizes rendered by one
 * persistent launch.  rgba_out receives the views' [H][W][4] images back to
 * back, aux_out (optional) their [H][W][8 + aux_dim] aux images back to back.
 * Images equal rmesh_forward_tiled's per view.  rmesh_backward does not
 * follow this call (it follows a single-view rmesh_forward_tiled). */
RMESH_API int rmesh_forward_views(RmeshCtx* ctx, const RmeshCamera* cams, int32_t n_views, float* rgba_out,
                                  float* aux_out);

/* backward, lib.rs:1894-2031: must follow rmesh_forward_tiled on the same context;
 * reuses that call's sorted tile lists and image.  Outputs (any may be NULL):
 * d_vertices [3N], d_densities [M], d_base_colors [3M], d_color_grads [3M]. */
RMESH_API int rmesh_backward(RmeshCtx* ctx, const float* dl_d_image, float* d_vertices, float* d_densities,
                   float* d_base_colors, float* d_color_grads);

/* backward with the custom aux channels' gradient: the dl_d_aux argument and
 * d_aux_data output of the reference's backward (lib.rs:2043-2090, buffers
 * :702-704, 745-763).  dl_d_aux [H][W][aux_dim] (NULL: zero) is the loss
 * gradient of the aux image's custom channels (those after the eight fixed
 * ones of rmesh_forward_tiled's aux_out); d_aux_data [M][aux_dim] receives the
 * gradient of the per-tet aux data, and the other outputs also carry the aux
 * channels' optical-depth terms.  The aux channels composite as
 * aux += T * alpha * a[tet] (rasterize_compute.wgsl:458-462); the adjoint is
 * the exact derivative of that sum (its d_aux_data term is the reference's
 * backward_interval_tiled.wgsl:637-649).  Same rules as rmesh_backward;
 * a context with aux_dim 0 gives rmesh_backward's results. */
RMESH_API int rmesh_backward_aux(RmeshCtx* ctx, const float* dl_d_image, const float* dl_d_aux, float* d_vertices,
                                 float* d_densities, float* d_base_colors, float* d_color_grads,
                                 float* d_aux_data);

/* forward_error, lib.rs:1621-1710 (the kernel: crates/rmesh-error/src/wgsl/
 * error_tiled_compute.wgsl): per-tet error statistics over the tile lists of
 * the last rmesh_forward_tiled.  pixel_err, ssim_err [H*W]; outputs
 * tet_err [M][16] f32 (0 weight, 1 weight*L1, 2 weight*L1^2, 5 weight*SSIM,
 * 6..8 weight*entry point, 9..11 weight*exit point, 12 weight,
 * 13..15 weight*centroid; weight = T * optical depth) and tet_count [M][2]
 * i32 (covered pixels, max of int(65535 * weight)), cleared by the call. */
RMESH_API int rmesh_forward_error(RmeshCtx* ctx, const float* pixel_err, const float* ssim_err, float* tet_err,
                                  int32_t* tet_count);

/* train_step, lib.rs:2405-2636: forward, loss, adjoint, Adam on vertices,
 * densities and color_grads; step += 1.  gt_rgb [H][W][3].  *loss_out receives
 * sum over pixels and RGB of (r-gt)^2 / n_pixels (L2) or |r-gt| / n_pixels (L1);
 * the reference returns 0.0 here (its loss buffer is never written). */
RMESH_API int rmesh_train_step(RmeshCtx* ctx, const RmeshCamera* cam, const float* gt_rgb, float lr_verts,
                     float lr_dens, float lr_grads, int32_t loss_type, float* loss_out);

/* Multi-view training step (no reference counterpart): the gradient of the sum
 * of the per-view losses over n_views cameras, then ONE Adam update.
 * gt_rgb holds the views' [H][W][3] images back to back.  loss_out (optional)
 * receives n_views per-view losses. */
RMESH_API int rmesh_train_step_views(RmeshCtx* ctx, const RmeshCamera* cams, int32_t n_views, const float* gt_rgb,
                           const RmeshTrainOpts* opts, float* loss_out);

/* Data-parallel split of rmesh_train_step_views (no reference counterpart):
 * accumulate the gradient of this rank's views into the context's per-tet
 * gradient slots (zeroed first, no Adam); expose those slots (device memory,
 * n_floats = 20 * M, plus 3 * nc * M SH coefficient gradients after them in
 * an SH context) so the caller can sum them across ranks, e.g. with an
 * NCCL all-reduce; then apply one Adam update from the slots. */
RMESH_API int rmesh_accumulate_views(RmeshCtx* ctx, const RmeshCamera* cams, int32_t n_views, const float* gt_rgb,
                                     const RmeshTrainOpts* opts, float* loss_out);
RMESH_API int rmesh_grad_slots(RmeshCtx* ctx, float** device_ptr, uint64_t* n_floats);

/* Tile configurations (no reference counterpart; the reference fixes 12-pixel
 * tiles, lib.rs:442).  A configuration is a tile size (8, 12 or 16) and the
 * threads per tile: one per pixel rounded up to whole warps (64, 160, 256; pass
 * 0 for it) or twice that (128, 320, 512: the item-parallel phases of the tile
 * kernel get more threads and larger sub-batches, half as many tiles are
 * resident per SM).  The pair-sort key width follows from the tile count.
 * set_tile_config sets the default configuration; set_resolution_tile_config
 * gives views of width x height their own (tile_size 0 removes it), so one
 * multi-view step can run, e.g., its 256x256 views at tile 8 and the rest at
 * 12 (the views of each configuration form one persistent launch).
 * get_tile_config returns the configuration a view of that size would use
 * (width, height 0: the default). */
RMESH_API int rmesh_set_tile_config(RmeshCtx* ctx, int32_t tile_size, int32_t threads);
RMESH_API int rmesh_set_resolution_tile_config(RmeshCtx* ctx, int32_t width, int32_t height, int32_t tile_size,
                                               int32_t threads);
RMESH_API int rmesh_get_tile_config(RmeshCtx* ctx, int32_t width, int32_t height, int32_t* tile_size,
                                    int32_t* threads);

/* One measurement of rmesh_autotune: ms per batched forward + loss + adjoint
 * run of the views of width x height (0, 0: all views of the call; -1, -1:
 * all views with the per-resolution configurations chosen) at tile_size /
 * threads. */
typedef struct {
  int32_t width;
  int32_t height;
  int32_t tile_size;
  int32_t threads;
  float ms;
} RmeshTuneEntry;

/* Autotuner over the whole configuration grid (tile size x threads per tile):
 * times every configuration on all views (no Adam, so the parameters are
 * unchanged) and makes the fastest the default; with per_resolution != 0 and
 * several resolutions among the views, also times every configuration on the
 * views of each resolution, gives a resolution whose fastest configuration
 * differs its own, and keeps those overrides only if the mixed step beats the
 * best single configuration.  Every measurement goes to entries (up to
 * max_entries; *n_entries = how many were made).  Reference design input:
 * crates/rmesh-backward/examples/tile_size_sweep.rs:1-60. */
RMESH_API int rmesh_autotune(RmeshCtx* ctx, const RmeshCamera* cams, int32_t n_views, const float* gt_rgb,
                             const RmeshTrainOpts* opts, int32_t per_resolution, RmeshTuneEntry* entries,
                             int32_t max_entries, int32_t* n_entries);

/* Tile-size autotuner (no reference counterpart; the reference fixes 12):
 * times the batched forward + loss + adjoint of these views (no Adam, so the
 * parameters are unchanged) at tile sizes 8, 12 and 16 -- which also sets the
 * threads per tile (64, 160, 256) and the pair-sort key width -- keeps the
 * fastest and returns it in *tile_size_out; ms_out (optional, [3]) receives
 * the milliseconds per run of each size.  Clears per-resolution configurations;
 * rmesh_autotune searches the whole grid. */
RMESH_API int rmesh_autotune_tile_size(RmeshCtx* ctx, const RmeshCamera* cams, int32_t n_views, const float* gt_rgb,
                                       const RmeshTrainOpts* opts, int32_t* tile_size_out, float* ms_out);
RMESH_API int rmesh_apply_adam(RmeshCtx* ctx, const RmeshTrainOpts* opts);

/* ---- .rmesh scene decode -------------------------------------------------------
 * The packed sections of a .rmesh file (crates/rmesh-data/src/lib.rs:247-393;
 * the host parses the header and slices the decompressed bytes) -> the
 * renderer's fp32 buffers, decoded on the device: densities exp((u8-100)/20),
 * colour gradients f16 -> f32 (zeros when color_grads is NULL), SH
 * coefficients [M][3][nc] = mean + weights x basis (PCA), circumdata
 * [M][4] computed in double with the loader's degenerate-tet rules.  All
 * pointers are device memory of the current device; asynchronous on stream. */
typedef struct {
  uint64_t n_vertices;
  uint64_t n_tets;
  uint32_t sh_degree;          /* 0..3 */
  uint32_t k_components;       /* PCA components in the file (min(k, 3 nc) are stored) */
  const float* vertices;       /* [3N] */
  const uint32_t* indices;     /* [4M] */
  const uint8_t* log_densities;   /* [M] */
  const uint16_t* sh_mean;     /* [3 nc] f16 */
  const uint16_t* sh_basis;    /* [k][3 nc] f16 */
  const uint16_t* sh_weights;  /* [M][k] f16 */
  const uint16_t* color_grads; /* [3M] f16 or NULL */
} RmeshPackedScene;
RMESH_API int rmesh_decode_scene(const RmeshPackedScene* scene, float* densities, float* color_grads,
                                 float* sh_coeffs, float* circumdata, void* stream);

/* ---- allocation-free tile count ---------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory (a per-frame visibility query in a viewer loop, where cudaMalloc and
 * cudaFree would synchronise the device; a caller with a fixed memory budget
 * that holds no context): the per-tet cull and conservative tile count of the
 * project stage (project_compute.wgsl:88-262, the values rmesh_debug_tiles_touched
 * reports after a single-view rmesh_forward_tiled) for one camera, plus the ids
 * of the tile-touching tets, with no context and no allocation.
 *  - All arrays are CUDA device (or managed) memory of the current device:
 *    vertices [3 * n_vertices], indices [4 * n_tets], densities [n_tets];
 *    outputs tiles_touched [n_tets] (by tet id), visible_tets [n_tets] (the
 *    first counts[0] entries are the tile-touching tet ids, ascending) and
 *    counts [2] (counts[1] receives device error bits: 2 = a bounded spin gave
 *    up, 4 = a vertex index >= n_vertices).  cam->cam_pos and c2w_intrinsics
 *    are not used.  tile_size 0 means 12.
 *  - n_tets above RMESH_STATIC_MAX_TETS returns RMESH_ERR_TOO_LARGE.
 *  - Asynchronous on `stream` (a cudaStream_t; NULL = the legacy default
 *    stream): read the outputs after synchronising it.
 *  - Scratch is one fixed 524,544-byte device array per device, shared by every
 *    call; each call clears what must start at zero on its stream.  Calls in
 *    flight at the same time on one device race on it: order them.  The first
 *    call on each device (with that device current) looks up the array's
 *    address and should come before any stream capture. */
#define RMESH_STATIC_MAX_TETS (1u << 24)
RMESH_API int rmesh_count_tiles_static(const float* vertices, uint64_t n_vertices, const uint32_t* indices,
                                       const float* densities, uint64_t n_tets, const RmeshCamera* cam,
                                       int32_t tile_size, uint32_t* tiles_touched, uint32_t* visible_tets,
                                       uint32_t* counts, void* stream);

/* ---- inspection (parity tests) --------------------------------------------- */
/* tiles_touched of the last forward, indexed by tet id ([M], single view). */
RMESH_API int rmesh_debug_tiles_touched(RmeshCtx* ctx, uint32_t* out);
/* sorted (tile id, tet id) slots of the last forward; *n receives the slot count
 * (sentinel slots carry tile 0xFFFFFFFF); at most cap entries are written. */
RMESH_API int rmesh_debug_pairs(RmeshCtx* ctx, uint32_t* tile_ids, uint32_t* tet_ids, uint64_t cap, uint64_t* n);
/* [start, end) per tile of the last forward ([2 * tiles]). */
RMESH_API int rmesh_debug_ranges(RmeshCtx* ctx, uint32_t* ranges, uint64_t n_tiles);

/* No reference counterpart: runs the path's two bounded waits (chained-scan
 * look-back, TMA mbarrier) on conditions that never resolve and returns, in
 * bits_out[0..1], the error bits each wait recorded after giving up (2 =
 * RMESH spin timeout).  The device stays usable; used by the failure tests. */
RMESH_API int rmesh_debug_timeouts(uint32_t* bits_out);

/* ---- profiling -------------------------------------------------------------- */
/* When enabled, CUDA events bracket each stage on the context stream; the
 * accumulated milliseconds are returned by rmesh_stage_times in the order
 * records, project, tet_sort, emit, pair_sort, ranges, composite, adam,
 * sh_adjoint (the SH colour adjoint; zero without SH colours).
 * ms_out has RMESH_N_STAGES entries; launches_out has RMESH_N_STAGES + 1
 * (per-stage span counts, then the number of kernels launched).  Both are
 * reset by the call. */
#define RMESH_N_STAGES 9
RMESH_API int rmesh_set_profiling(RmeshCtx* ctx, int32_t on);
RMESH_API int rmesh_stage_times(RmeshCtx* ctx, float* ms_out, int32_t* launches_out);

#ifdef __cplusplus
}
#endif

#endif /* RMESH_B200_H */
