// density_ctl.cu -- adaptive density control of 3DGSMR on the device: split,
// clone and prune of the Gaussian rows together with the Adam-state
// transplant, with no host synchronisation, so that a whole training
// iteration including a densification step stays one CUDA graph.
//
// Reference semantics (3DGS/3dgsVC/trainers/trainer.py:294-424 and
// gaussian/gaussian_model.py:85-222), applied to the live rows [0, n):
//   g    = |dL/dposition| (taken before gradient clipping, trainer.py:431-433)
//   smax = max_a exp(log_scale_a)
//   split = g > grad_thr & smax > scale_thr      (split branch if any and
//                                                  n + n_split <= max_points)
//   clone = g > grad_thr & smax <= scale_thr     (only without a split branch,
//                                                  with cloning enabled and
//                                                  n + n_clone <= max_points)
//   nothing at all when n >= max_points.
//   After the branch: prune = |rho| < opacity_thr | smax > max_scale, applied
//   when at least `min_keep` rows survive and one row is pruned.
// Row order is the reference's: split keeps the surviving rows in order and
// appends the first children of all parents, then the second children;
// clone appends one copy per parent; prune compacts in order.  Appended rows
// start with zero Adam moments, surviving rows carry theirs.
//
// The rows live in capacity-sized arrays; the live count is a device word.
// Rows past it are parked (zero moments, unit scale, identity rotation, zero
// density) and the voxelizer skips them (gsv_prepare_live).  Ranks come from
// one exclusive scan of a packed 64-bit flag (low word: survivor, high word:
// clone parent), and rows move through a scratch copy, so every step is a
// fixed sequence of launches whose work depends only on device data.
#include <cub/cub.cuh>

#include "gsv_common.cuh"

namespace {

constexpr int kBlock = 256;
constexpr int kCols = 15;  // 5 parameter tensors, their exp_avg and exp_avg_sq

enum Mode : int { kNone = 0, kSplit = 1, kClone = 2, kStop = 3 };

struct Counters {
    int32_t n0;       // live rows on entry
    int32_t n_split;  // split candidates among them
    int32_t n_clone;  // clone candidates among them
    int32_t n_keep;   // rows surviving the prune test (after the branch)
    int32_t n_prune;  // rows failing it
    int32_t pad[11];
};

struct Table {
    float* col[kCols];
    float* tmp[kCols];
    int width[kCols];
};

struct DensityLayout {
    size_t counters, flags, ranks, scan_tmp, tmp, total;
    size_t scan_tmp_bytes;
};

constexpr int kWidth[5] = {3, 3, 4, 1, 1};

DensityLayout density_layout(int64_t cap) {
    DensityLayout L{};
    size_t o = 0;
    L.counters = o;  o = gsv::align_up(o + sizeof(Counters));
    L.flags = o;     o = gsv::align_up(o + size_t(cap) * sizeof(int64_t));
    L.ranks = o;     o = gsv::align_up(o + size_t(cap) * sizeof(int64_t));
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<int64_t*>(nullptr),
                                  static_cast<int64_t*>(nullptr), int(cap > 0 ? cap : 1));
    L.scan_tmp_bytes = scan_bytes;
    L.scan_tmp = o;  o = gsv::align_up(o + scan_bytes);
    L.tmp = o;       o = gsv::align_up(o + size_t(cap) * 12 * 3 * sizeof(float));
    L.total = o;
    return L;
}

// Branch decision of the reference, from the candidate counts alone; every
// thread of every later launch evaluates it identically.
__device__ __forceinline__ int branch_mode(const Counters& c, const gsv_density_config& cfg, int64_t cap,
                                           bool* overflow) {
    *overflow = false;
    const int64_t n = c.n0;
    if (n >= cfg.max_points) return kStop;
    if (c.n_split > 0 && n + c.n_split <= cfg.max_points) {
        if (n + c.n_split > cap) {
            *overflow = true;
            return kStop;
        }
        return kSplit;
    }
    if (cfg.use_cloning && c.n_clone > 0 && n + c.n_clone <= cfg.max_points) {
        if (n + c.n_clone > cap) {
            *overflow = true;
            return kStop;
        }
        return kClone;
    }
    return kNone;
}

__device__ __forceinline__ int32_t rows_after_branch(const Counters& c, int mode) {
    return c.n0 + (mode == kSplit ? c.n_split : (mode == kClone ? c.n_clone : 0));
}

__device__ __forceinline__ bool prune_applies(const Counters& c, const gsv_density_config& cfg) {
    return c.n_keep >= cfg.min_keep && c.n_prune > 0;
}

__device__ __forceinline__ float max_scale_of(const float* ls) {
    return gsv::nanmax3(expf(ls[0]), expf(ls[1]), expf(ls[2]));
}

__device__ __forceinline__ void warp_count(bool pred, int32_t* counter) {
    const unsigned b = __ballot_sync(0xffffffffu, pred);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(counter, __popc(b));
}

// Candidates of the branch.  flags[i] = survivor-of-split | clone-parent << 32.
__global__ void __launch_bounds__(kBlock) k_classify(const int32_t* __restrict__ live, int64_t cap,
                                                     const float* __restrict__ pos_grad,
                                                     const float* __restrict__ log_scales, gsv_density_config cfg,
                                                     int64_t* __restrict__ flags, Counters* __restrict__ cnt) {
    const int32_t n = max(0, min(*live, int32_t(cap)));  // every later launch works on rows < n0 <= cap
    const int64_t base = int64_t(blockIdx.x) * blockDim.x;
    if (base == 0 && threadIdx.x == 0) cnt->n0 = n;
    for (int64_t i = base + threadIdx.x; i - threadIdx.x < cap; i += int64_t(gridDim.x) * blockDim.x) {
        bool split = false, clone = false;
        const bool active = i < n && i < cap;
        if (active) {
            const float gx = pos_grad[i * 3], gy = pos_grad[i * 3 + 1], gz = pos_grad[i * 3 + 2];
            const float g = sqrtf(__fmaf_rn(gz, gz, __fmaf_rn(gy, gy, __fmul_rn(gx, gx))));
            const float smax = max_scale_of(log_scales + i * 3);
            const bool high = g > cfg.grad_threshold;
            split = high && smax > cfg.scale_threshold;
            clone = high && smax <= cfg.scale_threshold;
        }
        if (i < cap) flags[i] = int64_t(active && !split) | (int64_t(clone) << 32);
        warp_count(split, &cnt->n_split);
        warp_count(clone, &cnt->n_clone);
    }
}

__device__ __forceinline__ void copy_row(const Table& t, int64_t src, float* const* dst_cols, int64_t dst) {
#pragma unroll
    for (int c = 0; c < kCols; ++c) {
        if (!t.col[c]) continue;
        const int w = t.width[c];
        for (int k = 0; k < w; ++k) dst_cols[c][dst * w + k] = t.col[c][src * w + k];
    }
}

__device__ __forceinline__ void restore_row(const Table& t, int64_t i) {
#pragma unroll
    for (int c = 0; c < kCols; ++c) {
        if (!t.col[c]) continue;
        const int w = t.width[c];
        for (int k = 0; k < w; ++k) t.col[c][i * w + k] = t.tmp[c][i * w + k];
    }
}

__device__ __forceinline__ void zero_moments(const Table& t, float* const* dst_cols, int64_t dst) {
#pragma unroll
    for (int c = 5; c < kCols; ++c) {
        if (!t.col[c]) continue;
        const int w = t.width[c];
        for (int k = 0; k < w; ++k) dst_cols[c][dst * w + k] = 0.0f;
    }
}

// Children of one split parent (gaussian_model.py:112-154).
__device__ void write_split_children(const Table& t, float* const* dst, int64_t i, int64_t a, int64_t b,
                                     const float* __restrict__ noise, const gsv_density_config& cfg) {
    const float* pos = t.col[0] + i * 3;
    const float* ls = t.col[1] + i * 3;
    const float* rot = t.col[2] + i * 4;
    float s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = expf(ls[k]);
    float pa[3], pb[3], cls[3];
    float dr = t.col[3][i], di = t.col[4][i];
    if (cfg.long_axis_split) {
        // longest axis (first maximum), child scales x0.5 on it and x0.85 on
        // the others, shift of child_scale * factor along the rotated axis
        int ax = 0;
        if (s[1] > s[ax]) ax = 1;
        if (s[2] > s[ax]) ax = 2;
        float cs[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) cs[k] = __fmul_rn(s[k], k == ax ? 0.5f : 0.85f);
        const float shift = __fmul_rn(cs[ax], cfg.long_axis_offset_factor);
        // quaternion_to_rotation_matrix (gaussian_model.py:12-19), column ax
        float n2 = __fmul_rn(rot[0], rot[0]);
        n2 = __fadd_rn(n2, __fmul_rn(rot[1], rot[1]));
        n2 = __fadd_rn(n2, __fmul_rn(rot[2], rot[2]));
        n2 = __fadd_rn(n2, __fmul_rn(rot[3], rot[3]));
        const float den = __fadd_rn(sqrtf(n2), 1e-8f);
        const float w = __fdiv_rn(rot[0], den), x = __fdiv_rn(rot[1], den);
        const float y = __fdiv_rn(rot[2], den), z = __fdiv_rn(rot[3], den);
        float r[3];
        if (ax == 0) {
            r[0] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(2.0f * y, y)), __fmul_rn(2.0f * z, z));
            r[1] = __fadd_rn(__fmul_rn(2.0f * x, y), __fmul_rn(2.0f * z, w));
            r[2] = __fsub_rn(__fmul_rn(2.0f * x, z), __fmul_rn(2.0f * y, w));
        } else if (ax == 1) {
            r[0] = __fsub_rn(__fmul_rn(2.0f * x, y), __fmul_rn(2.0f * z, w));
            r[1] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(2.0f * x, x)), __fmul_rn(2.0f * z, z));
            r[2] = __fadd_rn(__fmul_rn(2.0f * y, z), __fmul_rn(2.0f * x, w));
        } else {
            r[0] = __fadd_rn(__fmul_rn(2.0f * x, z), __fmul_rn(2.0f * y, w));
            r[1] = __fsub_rn(__fmul_rn(2.0f * y, z), __fmul_rn(2.0f * x, w));
            r[2] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(2.0f * x, x)), __fmul_rn(2.0f * y, y));
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float gs = __fmul_rn(r[k], shift);
            pa[k] = __fadd_rn(pos[k], gs);
            pb[k] = __fsub_rn(pos[k], gs);
            cls[k] = logf(__fadd_rn(cs[k], 1e-8f));
        }
        dr = __fmul_rn(dr, 0.6f);
        di = __fmul_rn(di, 0.6f);
    } else {
        // children ~ N(parent, (0.5 s)^2), scales s / 1.6 (torch divides by a
        // scalar as a product with its FP32 reciprocal)
        constexpr float kInv16 = 1.0f / 1.6f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pa[k] = __fadd_rn(pos[k], __fmul_rn(__fmul_rn(noise[i * 6 + k], s[k]), 0.5f));
            pb[k] = __fadd_rn(pos[k], __fmul_rn(__fmul_rn(noise[i * 6 + 3 + k], s[k]), 0.5f));
            cls[k] = logf(__fadd_rn(__fmul_rn(s[k], kInv16), 1e-8f));
        }
        dr = __fmul_rn(dr, 0.5f);
        di = __fmul_rn(di, 0.5f);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dst[0][a * 3 + k] = pa[k];
        dst[0][b * 3 + k] = pb[k];
        dst[1][a * 3 + k] = cls[k];
        dst[1][b * 3 + k] = cls[k];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        dst[2][a * 4 + k] = rot[k];
        dst[2][b * 4 + k] = rot[k];
    }
    dst[3][a] = dr;
    dst[3][b] = dr;
    dst[4][a] = di;
    dst[4][b] = di;
    zero_moments(t, dst, a);
    zero_moments(t, dst, b);
}

// Split: survivors and children into the scratch rows.  Clone: parents'
// densities halved in place and the copies appended in place.
__global__ void __launch_bounds__(kBlock) k_branch(Table t, int64_t cap, const Counters* __restrict__ cnt,
                                                   const int64_t* __restrict__ flags,
                                                   const int64_t* __restrict__ ranks,
                                                   const float* __restrict__ noise, gsv_density_config cfg) {
    const Counters c = *cnt;
    bool overflow;
    const int mode = branch_mode(c, cfg, cap, &overflow);
    if (mode != kSplit && mode != kClone) return;
    const int64_t n = c.n0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t f = flags[i];
        const int64_t r = ranks[i];
        if (mode == kSplit) {
            const int64_t keep_rank = r & 0xffffffffll;
            if (f & 1) {
                copy_row(t, i, t.tmp, keep_rank);
            } else {
                const int64_t n_keep = n - c.n_split;
                const int64_t child = i - keep_rank;  // rank among the parents
                write_split_children(t, t.tmp, i, n_keep + child, n_keep + c.n_split + child, noise, cfg);
            }
        } else if (f >> 32) {
            const int64_t dst = n + (r >> 32);
            const float dr = __fmul_rn(t.col[3][i], 0.5f), di = __fmul_rn(t.col[4][i], 0.5f);
            t.col[3][i] = dr;
            t.col[4][i] = di;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                t.col[0][dst * 3 + k] = t.col[0][i * 3 + k];
                t.col[1][dst * 3 + k] = logf(__fadd_rn(expf(t.col[1][i * 3 + k]), 1e-8f));
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) t.col[2][dst * 4 + k] = t.col[2][i * 4 + k];
            t.col[3][dst] = dr;
            t.col[4][dst] = di;
            zero_moments(t, t.col, dst);
        }
    }
}

// Split: scratch rows back over the live rows.
__global__ void __launch_bounds__(kBlock) k_split_commit(Table t, int64_t cap, const Counters* __restrict__ cnt,
                                                         gsv_density_config cfg) {
    const Counters c = *cnt;
    bool overflow;
    if (branch_mode(c, cfg, cap, &overflow) != kSplit) return;
    const int64_t rows = rows_after_branch(c, kSplit);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows; i += int64_t(gridDim.x) * blockDim.x)
        restore_row(t, i);
}

// Prune test on the rows after the branch; flags[i] = survivor.
__global__ void __launch_bounds__(kBlock) k_classify_prune(Table t, int64_t cap, Counters* __restrict__ cnt,
                                                           gsv_density_config cfg, int64_t* __restrict__ flags) {
    const Counters c = *cnt;
    bool overflow;
    const int mode = branch_mode(c, cfg, cap, &overflow);
    if (mode == kStop) return;
    const int64_t rows = rows_after_branch(c, mode);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i - threadIdx.x < rows;
         i += int64_t(gridDim.x) * blockDim.x) {
        bool keep = false, prune = false;
        if (i < rows) {
            const float smax = max_scale_of(t.col[1] + i * 3);
            const float mag = hypotf(t.col[3][i], t.col[4][i]);  // torch.abs of the complex density
            prune = mag < cfg.opacity_threshold || smax > cfg.max_scale;
            keep = !prune;
            flags[i] = int64_t(keep);
        }
        warp_count(keep, &cnt->n_keep);
        warp_count(prune, &cnt->n_prune);
    }
}

__global__ void __launch_bounds__(kBlock) k_prune_scatter(Table t, int64_t cap, const Counters* __restrict__ cnt,
                                                          gsv_density_config cfg, const int64_t* __restrict__ flags,
                                                          const int64_t* __restrict__ ranks) {
    const Counters c = *cnt;
    bool overflow;
    const int mode = branch_mode(c, cfg, cap, &overflow);
    if (mode == kStop || !prune_applies(c, cfg)) return;
    const int64_t rows = rows_after_branch(c, mode);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows; i += int64_t(gridDim.x) * blockDim.x)
        if (flags[i]) copy_row(t, i, t.tmp, ranks[i]);
}

__device__ __forceinline__ void park_row(const Table& t, int64_t i) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t.col[0][i * 3 + k] = 0.0f;
        t.col[1][i * 3 + k] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) t.col[2][i * 4 + k] = k == 0 ? 1.0f : 0.0f;
    t.col[3][i] = 0.0f;
    t.col[4][i] = 0.0f;
    zero_moments(t, t.col, i);
}

// Prune: scratch rows back, vacated rows parked.  Last launch of the call:
// block 0 publishes the new live count and the report.
__global__ void __launch_bounds__(kBlock) k_prune_commit(Table t, int64_t cap, const Counters* __restrict__ cnt,
                                                         gsv_density_config cfg, int32_t* __restrict__ live,
                                                         int32_t* __restrict__ report) {
    const Counters c = *cnt;
    bool overflow;
    const int mode = branch_mode(c, cfg, cap, &overflow);
    const bool pruned = mode != kStop && prune_applies(c, cfg);
    const int64_t rows = mode == kStop ? c.n0 : rows_after_branch(c, mode);
    const int64_t out = pruned ? c.n_keep : rows;
    if (pruned) {
        for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows;
             i += int64_t(gridDim.x) * blockDim.x) {
            if (i < out) restore_row(t, i);
            else park_row(t, i);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int32_t fl = 0;
        if (mode == kSplit) fl |= GSV_DENSITY_SPLIT;
        if (mode == kClone) fl |= GSV_DENSITY_CLONE;
        if (pruned) fl |= GSV_DENSITY_PRUNE;
        if (overflow) fl |= GSV_DENSITY_ROW_OVERFLOW;
        report[0] = fl;
        report[1] = mode == kSplit ? c.n_split : 0;
        report[2] = mode == kClone ? c.n_clone : 0;
        report[3] = pruned ? c.n_prune : 0;
        *live = int32_t(out);
    }
}

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with a
// Weyl-sequence key schedule.
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u, kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kM0 * c.x, hi0 = __umulhi(kM0, c.x);
        const uint32_t lo1 = kM1 * c.z, hi1 = __umulhi(kM1, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += kW0;
        k1 += kW1;
    }
    return c;
}

// uniform in (0, 1): (x + 1/2) 2^-32
__device__ __forceinline__ float unit_open(uint32_t x) {
    return __fmul_rn(__fadd_rn(float(x >> 8), 0.5f), 1.0f / 16777216.0f);
}

// Four standard normals per Philox block (Box-Muller), block q of stream
// *counter; the last launch advances the stream.
__global__ void __launch_bounds__(kBlock) k_normal_fill(float* __restrict__ out, int64_t count, uint64_t seed,
                                                        const int64_t* __restrict__ counter) {
    const uint64_t stream = uint64_t(*counter);
    const int64_t blocks = (count + 3) / 4;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < blocks;
         q += int64_t(gridDim.x) * blockDim.x) {
        const U4 r = philox4x32_10(U4{uint32_t(q), uint32_t(uint64_t(q) >> 32), uint32_t(stream),
                                      uint32_t(stream >> 32)},
                                   uint32_t(seed), uint32_t(seed >> 32));
        float z[4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float u1 = unit_open(h ? r.z : r.x), u2 = unit_open(h ? r.w : r.y);
            const float rad = sqrtf(-2.0f * logf(u1));
            float sn, cs;
            sincospif(2.0f * u2, &sn, &cs);
            z[2 * h] = rad * cs;
            z[2 * h + 1] = rad * sn;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (q * 4 + k < count) out[q * 4 + k] = z[k];
    }
}

__global__ void k_advance(int64_t* counter) { *counter += 1; }

int grid_of(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (n + kBlock - 1) / kBlock;
    return int(want < 1 ? 1 : (want > int64_t(sms) * 8 ? int64_t(sms) * 8 : want));
}

}  // namespace

extern "C" {

size_t gsv_density_workspace_bytes(int64_t capacity) {
    if (capacity <= 0 || capacity >= int64_t(INT32_MAX)) return 0;
    return density_layout(capacity).total;
}

int gsv_density_control(const gsv_density_rows* rows, const float* pos_grad, const float* noise,
                        const gsv_density_config* cfg, int32_t* live, int32_t* report, void* ws, size_t ws_bytes,
                        void* stream) {
    if (!rows || !cfg || !pos_grad || !live || !report || !ws) return GSV_ERR_INVALID_ARGUMENT;
    const int64_t cap = rows->capacity;
    if (cap <= 0 || cap >= int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    if (!rows->positions || !rows->log_scales || !rows->rotations || !rows->density_r || !rows->density_i)
        return GSV_ERR_INVALID_ARGUMENT;
    if (!cfg->long_axis_split && !noise) return GSV_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 5; ++k)
        if ((rows->exp_avg[k] == nullptr) != (rows->exp_avg_sq[k] == nullptr)) return GSV_ERR_INVALID_ARGUMENT;
    const DensityLayout L = density_layout(cap);
    if (ws_bytes < L.total) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(ws);
    Counters* cnt = reinterpret_cast<Counters*>(base + L.counters);
    int64_t* flags = reinterpret_cast<int64_t*>(base + L.flags);
    int64_t* ranks = reinterpret_cast<int64_t*>(base + L.ranks);

    Table t{};
    float* params[5] = {rows->positions, rows->log_scales, rows->rotations, rows->density_r, rows->density_i};
    float* tmp = reinterpret_cast<float*>(base + L.tmp);
    size_t off = 0;
    for (int k = 0; k < 5; ++k) {
        const int w = kWidth[k];
        t.col[k] = params[k];
        t.col[5 + k] = rows->exp_avg[k];
        t.col[10 + k] = rows->exp_avg_sq[k];
        t.width[k] = t.width[5 + k] = t.width[10 + k] = w;
        for (int j = 0; j < 3; ++j) {
            const int c = k + 5 * j;
            if (!t.col[c]) continue;
            t.tmp[c] = tmp + off;
            off += size_t(cap) * w;
        }
    }
    const gsv_density_config c = *cfg;
    const int grid = grid_of(cap);
    GSV_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(Counters), st));
    k_classify<<<grid, kBlock, 0, st>>>(live, cap, pos_grad, rows->log_scales, c, flags, cnt);
    GSV_LAUNCH_CHECK();
    size_t scan_bytes = L.scan_tmp_bytes;
    GSV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(base + L.scan_tmp, scan_bytes, flags, ranks, int(cap), st));
    k_branch<<<grid, kBlock, 0, st>>>(t, cap, cnt, flags, ranks, noise, c);
    GSV_LAUNCH_CHECK();
    k_split_commit<<<grid, kBlock, 0, st>>>(t, cap, cnt, c);
    GSV_LAUNCH_CHECK();
    k_classify_prune<<<grid, kBlock, 0, st>>>(t, cap, cnt, c, flags);
    GSV_LAUNCH_CHECK();
    GSV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(base + L.scan_tmp, scan_bytes, flags, ranks, int(cap), st));
    k_prune_scatter<<<grid, kBlock, 0, st>>>(t, cap, cnt, c, flags, ranks);
    GSV_LAUNCH_CHECK();
    k_prune_commit<<<grid, kBlock, 0, st>>>(t, cap, cnt, c, live, report);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_normal_fill(float* out, int64_t count, uint64_t seed, int64_t* counter, void* stream) {
    if (count < 0 || (count > 0 && !out) || !counter) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (count > 0) {
        k_normal_fill<<<grid_of((count + 3) / 4), kBlock, 0, st>>>(out, count, seed, counter);
        GSV_LAUNCH_CHECK();
    }
    k_advance<<<1, 1, 0, st>>>(counter);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
