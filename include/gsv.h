/*
 * gsv.h -- C ABI of the B200 (sm_100a) complex-Gaussian tile voxelizer.
 *
 * Plain pointers, sizes and a CUDA stream handle; no torch types.  Every
 * device pointer is caller-owned.  Every entry point only enqueues work on
 * `stream` (no host synchronisation) unless its comment says otherwise, so a
 * sequence of calls can be captured in a CUDA graph.
 *
 * Reference interfaces replaced (paths relative to the 3DGSMR project root,
 * V = 3DGS/3dgsVC):
 *   gsv_tile_forward            V/gaussian/cuda_ext/tile_voxelize_cuda.cpp:5-16,33-34
 *                               (tile_voxelize_forward_cuda, tile_voxelize_cuda_kernel.cu:262-300)
 *   gsv_tile_backward           V/gaussian/cuda_ext/tile_voxelize_cuda.cpp:18-31,35
 *                               (tile_voxelize_backward_cuda, tile_voxelize_cuda_kernel.cu:302-349)
 *   gsv_build_tile_pairs_count  V/gaussian/tile_voxelizer.py:87-118  (build_tile_pairs, up to the
 *                               host read of the pair total)
 *   gsv_build_tile_pairs_fill   V/gaussian/tile_voxelizer.py:120-162 (build_tile_pairs, rest)
 *   gsv_prepare / gsv_bin       V/gaussian/tile_voxelizer.py:282-293 (TileVoxelizer.forward
 *                               preprocess + binning, fused)
 *   gsv_forward                 V/gaussian/tile_voxelizer.py:296-309 (_TileVoxelizeCUDA.forward)
 *   gsv_backward                V/gaussian/tile_voxelizer.py:188-207 (_TileVoxelizeCUDA.backward)
 *                               fused with the torch autograd chain of :284-290 and :77-84
 *
 * Conventions
 *   - Volumes are (D,H,W) row-major.  Native volumes are complex64
 *     (interleaved re,im float pairs); the reference-compatible entry points
 *     use two float planes as the reference extension does.
 *   - positions [n,3] in [-1,1] (axis order d,h,w), scales [n,3] (the
 *     exp of the log-scale parameter, a fraction of the half extent),
 *     rotations [n,4] (w,x,y,z, unnormalised), density re/im [n]:
 *     the parameter layout of V/gaussian/gaussian_model.py:38-68.
 *   - Return value: a gsv_status.  Launch and argument errors are reported
 *     immediately; data-dependent conditions found on the device
 *     (capacity overflow, empty boxes) are latched in the workspace status
 *     word and read back with gsv_read_status.
 */
#ifndef GSV_H_
#define GSV_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GSV_API __attribute__((visibility("default")))
#else
#define GSV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GSV_ABI_VERSION 4

typedef enum gsv_status {
    GSV_OK = 0,
    GSV_ERR_INVALID_ARGUMENT = 1, /* bad shape, size, null pointer or workspace too small */
    GSV_ERR_CAPACITY = 2,         /* more (tile, Gaussian) pairs than the pair capacity */
    GSV_ERR_CUDA = 3,             /* a CUDA runtime call or launch failed */
    GSV_ERR_EMPTY_BOX = 4,        /* a Gaussian's tile box is empty (negative radius) */
    GSV_ERR_TOO_MANY_PAIRS = 5    /* pair total exceeds INT32_MAX (int32 tile ranges) */
} gsv_status;

/* Device-latched status bits (gsv_read_status). */
#define GSV_FLAG_CAPACITY_OVERFLOW 0x1
#define GSV_FLAG_EMPTY_BOX 0x2
#define GSV_FLAG_TOO_MANY_PAIRS 0x4
#define GSV_FLAG_SCAN_STALLED 0x8 /* a bounded wait of the preprocess's pair-count scan ran out */

/* Backward options. */
#define GSV_BACKWARD_DETERMINISTIC 0x1 /* fixed-order reduction: bitwise reproducible gradients */

typedef struct gsv_shape {
    int32_t d, h, w;   /* volume extent in voxels */
    int32_t tile_size; /* cubic binning tile edge (the reference's `tile_size`) */
} gsv_shape;

typedef struct gsv_params { /* device pointers, FP32, contiguous */
    const float* positions;
    const float* scales;
    const float* rotations;
    const float* density_r;
    const float* density_i;
    int64_t n;
} gsv_params;

typedef struct gsv_grads { /* device pointers, FP32, contiguous; fully overwritten */
    float* positions;
    float* scales;
    float* rotations;
    float* density_r;
    float* density_i;
} gsv_grads;

/* ---- library ---------------------------------------------------------- */

GSV_API int gsv_abi_version(void);
GSV_API const char* gsv_status_string(int status);
/* Text of the last CUDA failure seen by this thread (GSV_ERR_CUDA). */
GSV_API const char* gsv_last_error(void);
/* Number of tiles, ceil(d/ts)*ceil(h/ts)*ceil(w/ts); -1 for an invalid shape. */
GSV_API int64_t gsv_num_tiles(gsv_shape shape);

/* ---- workspace sizing ------------------------------------------------- */

/* Per-Gaussian / per-tile workspace (records, boxes, offsets, tile ranges,
 * gradient accumulators, status word). */
GSV_API size_t gsv_gauss_workspace_bytes(int64_t n, gsv_shape shape);
/* Per-pair workspace for `capacity` pairs (sort keys/values, sort scratch,
 * and the per-pair partials of the deterministic backward when
 * `flags & GSV_BACKWARD_DETERMINISTIC`). */
GSV_API size_t gsv_pair_workspace_bytes(int64_t capacity, gsv_shape shape, int flags);

/* ---- fused native path ------------------------------------------------ */

/* Preprocess every Gaussian (center, quadratic form, 3-sigma box), count its
 * tiles and scan the counts.  If `total_pairs_host` is non-NULL the pair
 * total is copied back and the stream is SYNCHRONISED (the reference's
 * `.item()` at tile_voxelizer.py:118); pass NULL to stay asynchronous. */
GSV_API int gsv_prepare(const gsv_params* params, gsv_shape shape, void* ws_gauss, size_t ws_gauss_bytes,
                int64_t* total_pairs_host, void* stream);

/* gsv_prepare over capacity-sized parameter rows of which only the first
 * `*live` (a device int32, read on the stream) are Gaussians: the other rows
 * get no tiles and contribute nothing, and their gradients are zero.  Used
 * with gsv_density_control, which changes the live count on the device. */
GSV_API int gsv_prepare_live(const gsv_params* params, const int32_t* live, gsv_shape shape, void* ws_gauss,
                             size_t ws_gauss_bytes, int64_t* total_pairs_host, void* stream);

/* Sort the (tile, Gaussian) pairs of the last gsv_prepare / gsv_prepare_live
 * on this workspace by tile (stable: ascending Gaussian id within a tile)
 * and build the per-tile ranges.  If the pair total exceeds `capacity` only
 * `capacity` pairs are kept and GSV_FLAG_CAPACITY_OVERFLOW is latched.  May
 * be called again after one preprocess (e.g. with a larger capacity).
 * Two sorts give the same lists: a counting sort over per-row tile counts
 * the preprocess writes when the grid has at most 3072 tiles and
 * ceil((n+1)/256)*4 rows x tiles <= 2^22 (three launches, no pair
 * keys), else an emit + radix sort + range pass.  gsv_bin picks the first
 * where it applies. */
#define GSV_BIN_AUTO 0
#define GSV_BIN_RADIX 1    /* always the radix sort */
#define GSV_BIN_COUNTING 2 /* the counting sort; GSV_ERR_INVALID_ARGUMENT where it does not apply */
GSV_API int gsv_bin(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, size_t ws_pairs_bytes,
            int64_t capacity, void* stream);
GSV_API int gsv_bin_ex(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, size_t ws_pairs_bytes,
                       int64_t capacity, int mode, void* stream);

/* Pointers to the tile ranges (int32 [T,2], empty tiles (0,0)) and the
 * sorted pair ids (int32 [capacity]) held inside the workspaces. */
GSV_API int gsv_bin_views(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, int64_t capacity,
                  int32_t** tile_ranges, int32_t** pair_ids);

/* Device addresses of the latched status flags (int32) and of the pair
 * total (int64) inside ws_gauss, for asynchronous checks (e.g. a copy to
 * pinned host memory captured in a CUDA graph). */
GSV_API int gsv_status_views(gsv_shape shape, int64_t n, void* ws_gauss, int32_t** flags,
                             int64_t** total_pairs);

/* Read the pair total and latched flags (SYNCHRONISES the stream). */
GSV_API int gsv_read_status(gsv_shape shape, int64_t n, const void* ws_gauss, int64_t* total_pairs,
                    int32_t* flags, void* stream);

/* volume: complex64 [d*h*w], fully overwritten (tiles without Gaussians
 * are written as zeros). */
GSV_API int gsv_forward(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs,
                int64_t capacity, float* volume, void* stream);

/* grad_volume: complex64 [d*h*w] (dL/dRe, dL/dIm).  Writes dL/d(positions,
 * scales, rotations, density_r, density_i).  `flags`: GSV_BACKWARD_*. */
GSV_API int gsv_backward(const gsv_params* params, gsv_shape shape, void* ws_gauss, void* ws_pairs,
                 int64_t capacity, const float* grad_volume, const gsv_grads* grads, int flags,
                 void* stream);

/* ---- batched persistent launches (many volumes, one launch) ---------- */

/* No counterpart in the reference (the batched multi-volume launch is an
 * addition).  One entry per volume, each already prepared and binned with
 * gsv_prepare / gsv_bin into its own workspaces (tile edge 8). */
typedef struct gsv_batch_item {
    gsv_shape shape;
    gsv_params params;        /* read by the backward (scales, rotations) */
    const void* ws_gauss;
    const void* ws_pairs;
    int64_t capacity;
    float* volume;            /* forward output, complex64 */
    const float* grad_volume; /* backward input, complex64 */
    gsv_grads grads;          /* backward outputs */
    int32_t chunk;            /* Gaussians per warp chunk, 1..32 (0 = 32) */
} gsv_batch_item;

GSV_API size_t gsv_batch_workspace_bytes(int count);
/* Upload the descriptor table of `count` volumes into ws_batch (device);
 * SYNCHRONISES the stream.  `flags`: GSV_BACKWARD_DETERMINISTIC must match
 * the flags the pair workspaces were sized with. */
GSV_API int gsv_batch_setup(const gsv_batch_item* items, int count, int flags, void* ws_batch, size_t ws_bytes,
                            void* stream);
/* One persistent launch over every tile of every volume (CTAs pull tiles
 * from an atomic counter); asynchronous, capturable. */
GSV_API int gsv_forward_batched(void* ws_batch, int count, void* stream);
/* Zeroing, one persistent backward launch, one finalize launch. */
GSV_API int gsv_backward_batched(void* ws_batch, int count, int flags, void* stream);

/* ---- execution tuning (results do not depend on it) ------------------ */

/* No counterpart in the reference.  rows_per_lane: 2 = one CTA per 8^3 tile
 * (two 8-voxel rows per lane), 1 = one CTA per 4x8x8 half tile (one row per
 * lane; the deterministic backward always uses whole tiles).  chunk: number
 * of Gaussians a warp stages in shared memory at a time (1..32).  flags:
 * GSV_TUNE_NO_CULL turns off the extent cull (a Gaussian, or a 4x8x8 row
 * slot of it, whose conservative tight extent misses the CTA's voxels is
 * skipped; it contributes nothing there either way).  split: the
 * backward runs `split` CTAs per (half) tile, each walking every split-th
 * group of four list positions -- more CTAs for small volumes whose tiles
 * are too few to fill the GPU (the forward ignores it).  Tile edge 8 only;
 * other tile edges ignore it. */
#define GSV_TUNE_NO_CULL 0x1
typedef struct gsv_tuning {
    int32_t rows_per_lane;
    int32_t chunk;
    int32_t flags;
    int32_t split; /* backward, tile edge 8: CTAs sharing one (half) tile's Gaussian list, 1, 2 or 4 (0 = 1) */
} gsv_tuning;

/* gsv_forward / gsv_backward with an explicit execution shape (NULL =
 * defaults: rows_per_lane 2, chunk 32). */
GSV_API int gsv_forward_ex(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs,
                           int64_t capacity, float* volume, const gsv_tuning* tuning, void* stream);
GSV_API int gsv_backward_ex(const gsv_params* params, gsv_shape shape, void* ws_gauss, void* ws_pairs,
                            int64_t capacity, const float* grad_volume, const gsv_grads* grads, int flags,
                            const gsv_tuning* tuning, void* stream);

/* No counterpart in the reference: a census of the work the tile-8 render
 * kernels do on a binned problem (a diagnostic for the roofline; results
 * unchanged).  out: FOUR device uint64 counters, overwritten --
 *   [0] included candidates (Mahalanobis <= 9, voxel inside the volume),
 *   [1] candidates the kernels evaluate the quadratic for (voxels of the
 *       4x8x8 row slots the extent cull keeps),
 *   [2] lanes issued by the per-column exp / FMA blocks (32 per voxel column
 *       of a kept slot in which some lane is inside the cutoff),
 *   [3] kept slots without any included voxel.
 * tuning (may be NULL): only GSV_TUNE_NO_CULL is read.  Tile edge 8 only.
 * Asynchronous on `stream`. */
GSV_API int gsv_count_work(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs,
                           int64_t capacity, const gsv_tuning* tuning, unsigned long long* out, void* stream);

/* ---- reference-compatible binning ------------------------------------ */

/* build_tile_pairs(center_vox [n,3], radius_vox [n]) part 1: box + count +
 * scan.  Same synchronisation rule as gsv_prepare. */
GSV_API int gsv_build_tile_pairs_count(const float* center_vox, const float* radius_vox, int64_t n,
                               gsv_shape shape, void* ws_gauss, size_t ws_gauss_bytes,
                               int64_t* total_pairs_host, void* stream);
/* Part 2: writes tile_ranges int32 [T,2] and pair_ids int32 [capacity]
 * (capacity >= the pair total from part 1) exactly as the reference lays
 * them out, with ascending Gaussian id inside each tile. */
GSV_API int gsv_build_tile_pairs_fill(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs,
                              size_t ws_pairs_bytes, int64_t capacity, int32_t* tile_ranges,
                              int32_t* pair_ids, void* stream);

/* No counterpart in the reference.  Binning for callers that cannot allocate
 * device memory -- their GPU memory belongs to another allocator (a framework
 * that reserves the device up front, a process under a hard memory cap) or
 * they run on a path with a fixed memory plan.  Same outputs as
 * gsv_build_tile_pairs_count + gsv_build_tile_pairs_fill, but every scratch
 * buffer comes from one static device array of about 41 MiB that each GPU
 * loading this library holds until the process exits; the caller passes only
 * inputs and outputs.  Limits: n <= 262,144 Gaussians (else
 * GSV_ERR_INVALID_ARGUMENT) and at most 2,097,152 pairs (else
 * GSV_ERR_CAPACITY; GSV_ERR_CAPACITY also when the pair total exceeds
 * `pair_capacity`).  `*total_pairs` always receives the pair total; the call
 * synchronises `stream` once to read it.  The first call on a device (with
 * that device current) looks up the array's device address.  All calls share the array: calls that overlap on
 * the GPU race, so serialise them. */
GSV_API int gsv_build_tile_pairs_noalloc(const float* center_vox, const float* radius_vox, int64_t n,
                                         gsv_shape shape, int32_t* tile_ranges, int32_t* pair_ids,
                                         int64_t pair_capacity, int64_t* total_pairs, void* stream);

/* ---- learned warm start: BF16 tensor-core GEMM (tcgen05, sm_100a) ----- */

/* No counterpart in the reference (the warm-start MLP is an addition).
 * C[m,n] = sum_k A[m,k] B[n,k] with BF16 operands read through element
 * strides (A(m,k) = a[m*a_sm + k*a_sk], B(n,k) = b[n*b_sn + k*b_sk]) and FP32
 * accumulation in tensor memory; C(m,n) lands at index m*c_sm + n*c_sn.
 * epi: 0 = FP32 store of acc (+ bias[n] if bias), 1 = z_f32 = acc + bias,
 * out_bf16 = GELU(z), 2 = out_bf16 = acc * GELU'(z_f32), 3 = atomicAdd of
 * acc into out_f32 (required when splits > 1: K split across CTAs).
 * col_sum (optional, epi 2 with c_sn == 1 only): col_sum[n] += sum over m of
 * the BF16 output (the bias gradient of the layer), accumulated with
 * atomics; zero it first.  N must be a multiple of 16.  *error (device int)
 * becomes 1 if a wait on the tensor cores timed out. */
GSV_API int gsv_mlp_gemm(const void* a, long long a_sm, long long a_sk, const void* b, long long b_sn,
                         long long b_sk, int M, int N, int K, int splits, const float* bias, float* out_f32,
                         void* out_bf16, float* z_f32, long long c_sm, long long c_sn, int epi, float* col_sum,
                         int* error, void* stream);

/* Test hook for the time-out path of gsv_mlp_gemm: C = A B^T (A [M,K], B [N,K]
 * row-major BF16, C [M,N] FP32) with the tensor-core work of K stage
 * `skip_stage` (64 columns of K each, 0 <= skip_stage < ceil(K/64)) left out,
 * so that the wait on it runs out after `wait_limit` polls (1 .. 2^26).  Every
 * CTA then sets *error = 1, waits for the tensor-core work it did issue,
 * frees its tensor memory and returns without writing C; the stream stays
 * usable.  Not for computing anything. */
GSV_API int gsv_mlp_gemm_test_timeout(const void* a, const void* b, int M, int N, int K, float* out_f32,
                                      int skip_stage, long long wait_limit, int* error, void* stream);

/* ---- fused SENSE data term around the FFTs ---------------------------- */

/* Replace the elementwise torch ops of the plain loss's data term
 * (V/trainers/trainer.py:256-268, V/losses/losses.py:18-26):
 *   L = sum_c || M * fft3c(S_c x) - y_c ||^2,  fft3c = fftshift o fftn(ortho) o ifftshift,
 * with the FFTs left to the caller (torch.fft / cuFFT) and the shifts folded
 * into the indexing.  Complex arrays are interleaved complex64; x, M are
 * [d,h,w], S, y and the coil images [ncoils,d,h,w].
 *   gsv_sense_expand  : out = ifftshift(S x)                  (then out <- fftn(out))
 *   gsv_sense_residual: kspace holds fftn(out); *loss = L (device float, fixed-order sum)
 *                       and kspace <- 2 M R, the gradient of L w.r.t. it    (then ifftn)
 *   gsv_sense_adjoint : volume_grad = sum_c conj(S_c) fftshift-inverse(ifftn(2 M R))_c,
 *                       dL/dx in torch's complex-gradient convention.
 * ws: gsv_sense_workspace_bytes() bytes of device scratch for the loss sum. */
GSV_API size_t gsv_sense_workspace_bytes(void);
GSV_API int gsv_sense_expand(const float* volume, const float* coils, int32_t ncoils, int32_t d, int32_t h, int32_t w,
                             float* out, void* stream);
GSV_API int gsv_sense_residual(float* kspace, const float* mask, const float* measured, int32_t ncoils, int32_t d,
                               int32_t h, int32_t w, float* loss, void* ws, size_t ws_bytes, void* stream);
GSV_API int gsv_sense_adjoint(const float* kgrad_image, const float* coils, int32_t ncoils, int32_t d, int32_t h,
                              int32_t w, float* volume_grad, void* stream);
/* Magnitude total variation of the plain loss (V/losses/losses.py:18-26, used at
 * V/trainers/trainer.py:261-274):
 * *loss = sum over the three axes of | |x|[i + e_a] - |x|[i] | (device float,
 * fixed-order sum) and grad = dTV/dx in torch's complex convention, one pass.
 * ws as for gsv_sense_residual. */
GSV_API int gsv_tv_magnitude(const float* volume, int32_t d, int32_t h, int32_t w, float* loss, float* grad, void* ws,
                             size_t ws_bytes, void* stream);

/* ---- intensity-seeded initialisation -------------------------------- */

/* ---- adaptive density control on the device ---------------------------- */

/* trainer.py:294-424 (adaptive_density_control, _transplant_adam_state,
 * _rebuild_optimizer) with gaussian_model.py:85-222 (densify_and_split,
 * densify_and_clone, _update_params), applied in place to capacity-sized rows
 * whose live count is a device word, with no host synchronisation (CUDA-graph
 * capturable).  Rows past the live count are parked: zero moments, unit
 * scale, identity rotation, zero density; gsv_prepare_live skips them. */
typedef struct gsv_density_rows { /* device pointers, FP32, row-major [capacity, width] */
    float* positions;     /* width 3 */
    float* log_scales;    /* width 3 */
    float* rotations;     /* width 4 */
    float* density_r;     /* width 1 */
    float* density_i;     /* width 1 */
    float* exp_avg[5];    /* Adam first moments of the five tensors above, or all NULL */
    float* exp_avg_sq[5]; /* Adam second moments, or all NULL */
    int64_t capacity;
} gsv_density_rows;

typedef struct gsv_density_config {
    float grad_threshold;          /* |dL/dposition| > this: densify candidate */
    float scale_threshold;         /* max scale > this: split, else clone */
    float opacity_threshold;       /* |density| < this: prune */
    float max_scale;               /* max scale > this: prune */
    float long_axis_offset_factor; /* long-axis children shift (gaussian_model.py:119-131) */
    int32_t long_axis_split;       /* 1: long-axis children; 0: N(parent, (s/2)^2) children from `noise` */
    int32_t use_cloning;           /* clone branch enabled */
    int32_t min_keep;              /* prune only when at least this many rows survive (100) */
    int64_t max_points;            /* no densification at or beyond this many rows */
} gsv_density_config;

/* report[0] bits; report[1..3] = rows split, cloned, pruned. */
#define GSV_DENSITY_SPLIT 0x1
#define GSV_DENSITY_CLONE 0x2
#define GSV_DENSITY_PRUNE 0x4
#define GSV_DENSITY_ROW_OVERFLOW 0x8 /* the branch needs more rows than `capacity`: nothing was changed */

GSV_API size_t gsv_density_workspace_bytes(int64_t capacity);
/* One density-control step.  pos_grad [capacity,3]: the position gradient
 * before clipping; noise [capacity,6]: standard normals for the two children
 * of a split parent row (first child columns 0-2, second 3-5), unused with
 * long_axis_split; live: device int32, read and updated; report: device
 * int32[4], written. */
GSV_API int gsv_density_control(const gsv_density_rows* rows, const float* pos_grad, const float* noise,
                                const gsv_density_config* cfg, int32_t* live, int32_t* report, void* ws,
                                size_t ws_bytes, void* stream);

/* `count` standard normals (Philox4x32-10 with Box-Muller) of stream
 * `*counter` (a device int64, read on the stream) under key `seed`, then
 * *counter += 1: a graph replay draws a fresh stream, and restoring the
 * counter replays the same draws.  The split noise of gsv_density_control
 * (torch.randn_like at gaussian_model.py:135-136). */
GSV_API int gsv_normal_fill(float* out, int64_t count, uint64_t seed, int64_t* counter, void* stream);

/* V/data/mask_generator.py:241-390 (_generate_poisson_mask_heuristic), for
 * `count` masks in one launch: variable-density Poisson-disc (ky, kz) masks
 * of ny x nz pixels (ny*nz <= 196608).  radius [ny*nz] FP64: the exclusion
 * radius per pixel (the reference's r_grid = 0.6 / sqrt(max(pdf, 1e-4)));
 * orders [count, ny*nz] int32: each mask's pixel visiting order (the
 * reference's np.random.permutation); calib: the calibration square's edge
 * (Python slice semantics around ny/2, nz/2); target: pixels to set
 * (int(ny*nz/accel)).  masks [count, ny*nz] int8 out; rounds [count] int32
 * out (may be NULL): parallel rounds used, -1 if that order is not a
 * permutation (its mask is then the calibration square).  Equal to the
 * reference's sequential pass for the same order.  ws: device scratch of
 * gsv_poisson_workspace_bytes(ny, nz, count) bytes (0: unsupported size). */
GSV_API size_t gsv_poisson_workspace_bytes(int32_t ny, int32_t nz, int32_t count);
GSV_API int gsv_poisson_masks(const double* radius, const int32_t* orders, int32_t ny, int32_t nz, int32_t calib,
                              int64_t target, int32_t count, int8_t* masks, int32_t* rounds, void* ws,
                              size_t ws_bytes, void* stream);

/* V/gaussian/gaussian_model.py:283-306 (_sampled_3nn_scale_init, a cKDTree on
 * the CPU): for n distinct seed voxels (flat row-major indices into the
 * (d,h,w) volume) with their FP32 normalised positions [n,3]
 * ((v + 0.5) / shape * 2 - 1 per axis), mean_distance[i] = FP32 mean of the
 * distances (FP64, rounded to FP32) from seed i to its 3 nearest other seeds,
 * at least 1e-6; the last found distance repeats when fewer than 3 other seeds
 * exist and a lone seed gets 1e-3.  grid: d*h*w int32 of device scratch.
 * Exact (grid shells, no approximation). */
GSV_API int gsv_knn3_mean_distance(const int64_t* voxels, const float* positions, int64_t n, int32_t d, int32_t h,
                                   int32_t w, int32_t* grid, float* mean_distance, void* stream);

/* ---- reference-compatible kernels (the pybind forward/backward) ------- */

/* centers [n,3] voxel units, cov_inv [n,3,3] normalised units (symmetric;
 * the symmetric part is used), density_r/i [n], tile_ranges [T,2],
 * pair_ids [P], half_shape [3] (device).  vol_r/vol_i [d*h*w] are fully
 * overwritten. */
GSV_API int gsv_tile_forward(const float* centers, const float* cov_inv, const float* density_r,
                     const float* density_i, const int32_t* tile_ranges, const int32_t* pair_ids,
                     const float* half_shape, int64_t n, int64_t num_tiles, int32_t tile_size,
                     int32_t d, int32_t h, int32_t w, float* vol_r, float* vol_i, void* stream);

/* Gradients w.r.t. centers [n,3], cov_inv [n,3,3] (symmetric), density_r,
 * density_i [n]; outputs are zeroed by the callee, then accumulated. */
GSV_API int gsv_tile_backward(const float* centers, const float* cov_inv, const float* density_r,
                      const float* density_i, const int32_t* tile_ranges, const int32_t* pair_ids,
                      const float* half_shape, const float* grad_vol_r, const float* grad_vol_i,
                      int64_t n, int64_t num_tiles, int32_t tile_size, int32_t d, int32_t h,
                      int32_t w, float* grad_centers, float* grad_cov_inv, float* grad_den_r,
                      float* grad_den_i, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSV_H_ */
