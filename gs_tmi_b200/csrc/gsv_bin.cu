// gsv_bin.cu -- preprocess and tile binning (device radix sort), sm_100a.
//
// Binning is bit-exact with build_tile_pairs (3DGS/3dgsVC/gaussian/
// tile_voxelizer.py:87-162): the FP32 center/radius follow :284-286 op for
// op, the voxel box uses floor/ceil + clamp (:97-105), the tile box integer
// division + clamp (:107-114), pairs are generated Gaussian-major in
// (d,h,w) raster order (:126-145) and stably sorted by tile id, so each
// tile's list is in ascending Gaussian id; empty tiles keep range (0,0)
// (:151-161).  Unlike the reference there is no host synchronisation unless
// the caller asks for the pair total.
#include <cub/cub.cuh>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "gsv_common.cuh"

using namespace gsv;

namespace {

thread_local char g_last_error[512] = {0};

constexpr int kMaxTilesPerAxis = 65535;  // box packing: 16 bits per field

struct ShapeInfo {
    int32_t d, h, w, ts, ntd, nth, ntw;
    int64_t ntiles;
    bool ok;
};

ShapeInfo shape_info(gsv_shape s) {
    ShapeInfo r{};
    r.ok = s.d > 0 && s.h > 0 && s.w > 0 && s.tile_size > 0 && s.d < (1 << 24) && s.h < (1 << 24) &&
           s.w < (1 << 24);
    if (!r.ok) return r;
    r.d = s.d; r.h = s.h; r.w = s.w; r.ts = s.tile_size;
    r.ntd = (s.d + s.tile_size - 1) / s.tile_size;
    r.nth = (s.h + s.tile_size - 1) / s.tile_size;
    r.ntw = (s.w + s.tile_size - 1) / s.tile_size;
    r.ok = r.ntd <= kMaxTilesPerAxis && r.nth <= kMaxTilesPerAxis && r.ntw <= kMaxTilesPerAxis;
    r.ntiles = int64_t(r.ntd) * r.nth * r.ntw;
    r.ok = r.ok && r.ntiles < (int64_t(1) << 30);
    return r;
}

int sort_end_bit(int64_t ntiles) {
    // keys are tile ids in [0, ntiles]; ntiles is the padding sentinel.
    int bits = 1;
    while ((int64_t(1) << bits) <= ntiles) ++bits;
    return bits;
}

// The preprocess scans the per-Gaussian pair counts in one pass (decoupled
// look-back): blocks of kPrepThreads Gaussians, one 64-bit look-back word per
// block after the Status struct, all cleared by the one memset of the status
// region that starts every preprocess.
constexpr int kPrepThreads = 256;
__host__ __device__ inline int64_t prep_blocks(int64_t n) { return (n + 1 + kPrepThreads - 1) / kPrepThreads; }

// Counting-sort binning, used when the tile count is small.  The pairs'
// final order is fixed by two facts: a tile's list holds its Gaussians in
// ascending id, and Gaussians are handled in rows of kCsSeg consecutive ids.
// k_prepare also writes, per row, how many of the row's pairs fall in each
// tile (rows x tiles bytes, "cs_mat": a row's count in one tile is at most
// kCsSeg; rows padded to whole words); k_colscan writes, per row and tile,
// the position of the row's first pair of that tile in the sorted output
// ("cs_pos": the column's exclusive prefix plus the tile's start, from a
// single-pass scan of the tile totals) and the tile ranges; k_scatter walks
// each row's Gaussians in id order and places their pairs.  The result
// equals the stable radix sort's, which larger problems keep.  The counts
// stay intact and k_scatter clears k_colscan's scan state, so binning may
// be repeated after one preprocess (e.g. with a larger capacity).
constexpr int kCsSeg = 64;                                  // Gaussians per row: two warps of k_prepare
constexpr int kCsRowsPerBlock = kPrepThreads / kCsSeg;      // rows per k_prepare block
// k_scatter keeps kCsRowsPerBlock x ntiles int32 in shared memory: at most 48 KB, the size a
// launch may use without a function attribute (none is set, also not inside a graph capture)
constexpr int64_t kCsMaxTiles = 3072;
constexpr int64_t kCsMaxCells = int64_t(1) << 22;           // rows x tiles: 4 MB of counts, 16 MB of positions
constexpr int kCsCols = 32, kCsRowGroups = 32;              // k_colscan block: 32 columns x 32 row groups
__host__ __device__ inline int64_t cs_rows(int64_t n) { return prep_blocks(n) * kCsRowsPerBlock; }
__host__ __device__ inline int64_t cs_col_blocks(int64_t ntiles) { return (ntiles + kCsCols - 1) / kCsCols; }
__host__ __device__ inline int64_t cs_mstride(int64_t ntiles) { return (ntiles + 3) & ~int64_t(3); }  // bytes per row
inline bool cs_eligible(int64_t n, int64_t ntiles) {
    return n > 0 && ntiles <= kCsMaxTiles && cs_rows(n) * ntiles <= kCsMaxCells;
}

// Status region: the Status word, the preprocess's look-back words (one per
// block), then k_colscan's (one per column block).  Status::pad[1] and
// pad[2] are the two launches' block-ticket counters.
__host__ __device__ inline size_t status_bytes(int64_t n, int64_t ntiles) {
    return sizeof(Status) + size_t(prep_blocks(n) + cs_col_blocks(ntiles)) * sizeof(unsigned long long);
}

GaussLayout gauss_layout(int64_t n, const ShapeInfo& si) {
    GaussLayout L{};
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int64_t*)nullptr, (int64_t*)nullptr,
                                  int(n + 1));
    L.scan_tmp_bytes = scan_bytes;
    size_t o = 0;
    L.rec = o;      o = align_up(o + size_t(n) * sizeof(Rec));
    L.ext = o;      o = align_up(o + size_t(n) * sizeof(float4));
    L.box = o;      o = align_up(o + size_t(n) * sizeof(int4));
    L.counts = o;   o = align_up(o + size_t(n + 1) * sizeof(int64_t));
    L.offsets = o;  o = align_up(o + size_t(n + 1) * sizeof(int64_t));
    L.scan_tmp = o; o = align_up(o + scan_bytes);
    L.ranges = o;   o = align_up(o + size_t(si.ntiles) * sizeof(int2));
    L.accum = o;    o = align_up(o + size_t(n) * kMomStride * sizeof(float));
    L.status = o;   o = align_up(o + status_bytes(n, si.ntiles));
    L.cs = cs_eligible(n, si.ntiles);
    L.cs_mat = o;   o = align_up(o + (L.cs ? size_t(cs_rows(n) * cs_mstride(si.ntiles)) : 0));
    L.cs_pos = o;   o = align_up(o + (L.cs ? size_t(cs_rows(n) * si.ntiles) * sizeof(int32_t) : 0));
    L.total = o;
    return L;
}

PairLayout pair_layout(int64_t cap, const ShapeInfo& si, int flags) {
    PairLayout L{};
    size_t sort_bytes = 0;
    const int end_bit = sort_end_bit(si.ntiles);
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const int32_t*)nullptr, (int32_t*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, int(cap > 0 ? cap : 1),
                                    0, end_bit);
    L.sort_tmp_bytes = sort_bytes;
    size_t o = 0;
    const size_t c = size_t(cap > 0 ? cap : 1);
    L.keys_in = o;  o = align_up(o + c * sizeof(int32_t));
    L.vals_in = o;  o = align_up(o + c * sizeof(int32_t));
    L.keys_out = o; o = align_up(o + c * sizeof(int32_t));
    L.vals_out = o; o = align_up(o + c * sizeof(int32_t));
    L.sort_tmp = o; o = align_up(o + sort_bytes);
    L.partials = o;
    if (flags & GSV_BACKWARD_DETERMINISTIC) o = align_up(o + c * kMomStride * sizeof(float));
    L.total = o;
    return L;
}

template <typename T>
T* at(void* base, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}
template <typename T>
const T* at(const void* base, size_t off) {
    return reinterpret_cast<const T*>(static_cast<const char*>(base) + off);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

struct DevShape {
    int32_t size[3];
    int32_t nt[3];
    int32_t ts;
    float shape_f[3];
    float hs[3];
    float ih[3];
};

DevShape dev_shape(const ShapeInfo& si) {
    DevShape s{};
    s.size[0] = si.d; s.size[1] = si.h; s.size[2] = si.w;
    s.nt[0] = si.ntd; s.nt[1] = si.nth; s.nt[2] = si.ntw;
    s.ts = si.ts;
    for (int a = 0; a < 3; ++a) {
        s.shape_f[a] = float(s.size[a]);
        s.hs[a] = s.shape_f[a] * 0.5f;
        s.ih[a] = 1.0f / s.hs[a];  // host IEEE division, same as the device __fdiv_rn
    }
    return s;
}

// Tile box of one Gaussian; returns the tile count (<= 0 for an empty box).
__device__ __forceinline__ int64_t tile_box(const DevShape& s, const float c[3], float r, int4* box) {
    int32_t tlo[3], na[3];
    int64_t cnt = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // (center_vox - r3).floor().int() / (center_vox + r3).ceil().int(), clamp (:97-105)
        int32_t lo = __float2int_rz(floorf(__fsub_rn(c[a], r)));
        int32_t hi = __float2int_rz(ceilf(__fadd_rn(c[a], r)));
        lo = min(max(lo, 0), s.size[a] - 1);
        hi = min(max(hi, 0), s.size[a] - 1);
        // // tile_size, clamp (:107-114); lo, hi >= 0 here so C division == floor division
        int32_t t0 = min(max(lo / s.ts, 0), s.nt[a] - 1);
        int32_t t1 = min(max(hi / s.ts, 0), s.nt[a] - 1);
        tlo[a] = t0;
        na[a] = t1 - t0 + 1;
        if (na[a] <= 0) cnt = 0;
        else cnt *= na[a];
    }
    box->x = tlo[0] | (tlo[1] << 16);
    box->y = tlo[2] | (max(na[0], 0) << 16);
    box->z = max(na[1], 0) | (max(na[2], 0) << 16);
    box->w = int32_t(cnt);
    return cnt;
}

// Look-back word of a block: flag in the top two bits, an int64 pair count
// below.  kLbAgg: the block's own total; kLbPre: the total of every block up
// to and including it.
constexpr unsigned long long kLbAgg = 1ull << 62, kLbPre = 2ull << 62, kLbVal = (1ull << 62) - 1;
constexpr int kLbSpinLimit = 1 << 22;  // polls of one predecessor's word before giving up

__device__ __forceinline__ unsigned long long lb_load(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void lb_store(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Decoupled look-back of scan block `bid`, run by all 32 lanes of one warp:
// publishes the block's total, walks back over the predecessors' words and
// returns the sum of every earlier block's total (the same in all lanes),
// after publishing its own inclusive prefix.  Lane l reads the word of block
// j - l, so one step covers 32 predecessors; the nearest inclusive prefix
// (kLbPre) in the window ends the walk, and every word in front of it must
// be published (flag set) before the window is summed, else the step is
// retried.  Block ids come from a ticket counter, so every block waited for
// has started.  Each retry is bounded: on time-out GSV_FLAG_SCAN_STALLED is
// latched and the block publishes what it has, so no later block waits the
// full limit again.
__device__ int64_t lookback(unsigned long long* lb, int64_t bid, int64_t block_tot, Status* status, int lane) {
    if (bid == 0) {
        if (lane == 0) lb_store(&lb[0], kLbPre | (unsigned long long)block_tot);
        return 0;
    }
    if (lane == 0) lb_store(&lb[bid], kLbAgg | (unsigned long long)block_tot);
    int64_t base = 0;
    int64_t j = bid - 1;  // the window's nearest predecessor
    int spins = 0;
    while (true) {
        const int64_t idx = j - lane;
        // before block 0 there is nothing: an inclusive prefix of zero
        const unsigned long long v = idx >= 0 ? lb_load(&lb[idx]) : kLbPre;
        const unsigned long long f = v & ~kLbVal;
        const unsigned pre = __ballot_sync(0xffffffffu, f == kLbPre);
        const int first = pre ? __ffs(pre) - 1 : 31;  // last lane of this step
        const unsigned upto = first == 31 ? 0xffffffffu : (2u << first) - 1u;
        const unsigned missing = __ballot_sync(0xffffffffu, f == 0) & upto;
        if (missing) {
            if (++spins > kLbSpinLimit) {
                if (lane == 0) atomicOr(&status->flags, GSV_FLAG_SCAN_STALLED);
                break;
            }
            continue;
        }
        spins = 0;
        int64_t part = ((upto >> lane) & 1u) ? int64_t(v & kLbVal) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        base += part;
        if (pre) break;
        j -= 32;
    }
    if (lane == 0) lb_store(&lb[bid], kLbPre | (unsigned long long)(base + block_tot));
    return base;
}

// Tile id of pair `c` (0-based, raster order) of a Gaussian's packed tile box.
__device__ __forceinline__ int32_t box_tile(const DevShape& s, int bx, int by, int bz, int32_t c) {
    const int32_t t0 = bx & 0xffff, t1 = (bx >> 16) & 0xffff, t2 = by & 0xffff;
    const int32_t n1 = bz & 0xffff, n2 = (bz >> 16) & 0xffff;
    const int32_t k = c % n2, r = c / n2;
    const int32_t jj = r % n1, i = r / n1;
    return ((t0 + i) * s.nt[1] + (t1 + jj)) * s.nt[2] + (t2 + k);
}

// box_tile for the counting sort, where the pair index and both box extents
// are below 4096 (they are at most the tile count, <= kCsMaxTiles): the two
// integer divisions become trunc((x + 0.5) * rcp(n)) in IEEE single
// precision, exact for 0 <= x < 4096 and 1 <= n <= 4096 (every pair checked
// by enumeration), a few instructions instead of about twenty each.  r1, r2:
// __frcp_rn of the box's n1, n2.
__device__ __forceinline__ int32_t small_div(int32_t x, float rcp_n) {
    return __float2int_rz(__fmul_rn(__fadd_rn(float(x), 0.5f), rcp_n));
}
__device__ __forceinline__ int32_t box_tile_small(const DevShape& s, int bx, int by, int bz, float r1, float r2,
                                                  int32_t c) {
    const int32_t t0 = bx & 0xffff, t1 = (bx >> 16) & 0xffff, t2 = by & 0xffff;
    const int32_t n1 = bz & 0xffff, n2 = (bz >> 16) & 0xffff;
    const int32_t r = small_div(c, r2), k = c - r * n2;
    const int32_t i = small_div(r, r1), jj = r - i * n1;
    return ((t0 + i) * s.nt[1] + (t1 + jj)) * s.nt[2] + (t2 + k);
}
__device__ __forceinline__ float box_rcp(int field) { return __frcp_rn(float(max(field & 0xffff, 1))); }

// Preprocess (center, radius, quadratic-form coefficients, tight extent, tile
// box) of one Gaussian per thread, the clearing of its backward moment
// accumulators, and the exclusive scan of the Gaussians'
// pair counts into `offsets` (offsets[n] = pair total) in the same launch.
// Blocks take their position in the scan from a counter in the status
// region, so every block a block waits for has already started; it waits
// only for its predecessors' published totals, each wait bounded (on
// time-out GSV_FLAG_SCAN_STALLED is latched and the block publishes anyway,
// so no later block waits the full limit again).  With `cs_mat` the block
// also counts its pairs per tile for each of its kCsRowsPerBlock rows and
// writes those rows of cs_mat.  A row's count in one tile is at most kCsSeg
// (< 256), so the counters are bytes, four to a word, in shared memory
// (dynamic: kCsRowsPerBlock x ceil(ntiles/4) words) and in cs_mat alike: the
// block's rows go out as the same words.
__global__ void __launch_bounds__(kPrepThreads) k_prepare(const float* __restrict__ pos,
                                                          const float* __restrict__ scl,
                                                          const float* __restrict__ rot,
                                                          const float* __restrict__ dr,
                                                          const float* __restrict__ di, int64_t n,
                                                          const int32_t* __restrict__ live, DevShape s,
                                                          Rec* __restrict__ recs, float4* __restrict__ ext,
                                                          int4* __restrict__ boxes,
                                                          int64_t* __restrict__ offsets, Status* status,
                                                          uint8_t* __restrict__ cs_mat, int32_t ntiles,
                                                          float* __restrict__ accum) {
    __shared__ int bid_s;
    __shared__ int64_t warp_tot[kPrepThreads / 32];
    __shared__ int64_t block_base;
    if (threadIdx.x == 0) bid_s = atomicAdd(&status->pad[1], 1);
    __syncthreads();
    const int64_t bid = bid_s;
    const int64_t g = bid * kPrepThreads + threadIdx.x;
    int64_t cnt = 0;
    int4 box = make_int4(0, 0, 0, 0);
    if (g < n) {  // the backward's moment accumulators start from zero
        float4* acc4 = reinterpret_cast<float4*>(accum + g * kMomStride);
        acc4[0] = acc4[1] = acc4[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (g < n && live && g >= int64_t(*live)) {  // parked row: no tiles, no contribution
        recs[g] = Rec{};
        ext[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        boxes[g] = make_int4(0, 0, 0, 0);
    } else if (g < n) {
        float p[3], sc[3], q[4];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            p[a] = pos[g * 3 + a];
            sc[a] = scl[g * 3 + a];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) q[k] = rot[g * 4 + k];
        float c[3], sv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            // center_vox = (positions + 1.0) * 0.5 * shape - 0.5   (:284)
            c[a] = __fsub_rn(__fmul_rn(__fmul_rn(__fadd_rn(p[a], 1.0f), 0.5f), s.shape_f[a]), 0.5f);
            sv[a] = __fmul_rn(sc[a], s.hs[a]);  // scale_vox (:285)
        }
        const float r = __fmul_rn(nanmax3(sv[0], sv[1], sv[2]), 3.0f);  // radius_vox (:286)
        float qc[6];
        qcoef_from_params(sc, q, s.ih, qc);
        Rec R;
        R.c0 = c[0]; R.c1 = c[1]; R.c2 = c[2];
        R.q00 = qc[0]; R.q01x2 = qc[1]; R.q02x2 = qc[2]; R.q11 = qc[3]; R.q12x2 = qc[4]; R.q22 = qc[5];
        R.rho_r = dr[g]; R.rho_i = di[g]; R.pad = 0.0f;
        recs[g] = R;
        ext[g] = tight_extent(qc);
        cnt = tile_box(s, c, r, &box);
        if (cnt <= 0) {
            atomicOr(&status->flags, GSV_FLAG_EMPTY_BOX);
            cnt = 0;
            box.w = 0;
        }
        boxes[g] = box;
    }
    // block-wide inclusive scan of the counts
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    int64_t warp_base = 0, block_tot = 0;
#pragma unroll
    for (int w = 0; w < kPrepThreads / 32; ++w) {
        if (w < warp) warp_base += warp_tot[w];
        block_tot += warp_tot[w];
    }
    if (warp == 0) {
        const int64_t base = lookback(reinterpret_cast<unsigned long long*>(status + 1), bid, block_tot, status, lane);
        if (lane == 0) block_base = base;
    }
    __syncthreads();
    if (g <= n) offsets[g] = block_base + warp_base + incl - cnt;
    if (cs_mat == nullptr) return;  // block-uniform

    // Per-row tile counts.  The warp's pairs occupy the block-local range
    // [wstart, wend), lane l's Gaussian the part starting at o; the lanes
    // stride over the range and find each pair's Gaussian by a shuffle
    // search over the 32 starts (zero-count lanes share their successor's
    // start and are never chosen).
    extern __shared__ uint32_t cs_hist[];  // [kCsRowsPerBlock][words]: byte counter of tile t in word t/4
    const int words = (ntiles + 3) >> 2;
    for (int i = threadIdx.x; i < kCsRowsPerBlock * words; i += kPrepThreads) cs_hist[i] = 0u;
    __syncthreads();
    {
        constexpr unsigned kAll = 0xffffffffu;
        const long long o = warp_base + incl - cnt;
        const long long wstart = __shfl_sync(kAll, o, 0);
        const long long wend = warp_base + warp_tot[warp];
        uint32_t* row = cs_hist + (warp * 32 / kCsSeg) * words;
        const float rcp1 = box_rcp(box.z), rcp2 = box_rcp(box.z >> 16);
        for (long long base = wstart; base < wend; base += 32) {
            const long long p = base + lane;
            int j = 0;  // largest j with o_j <= p
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const long long oj = __shfl_sync(kAll, o, j + step);
                if (oj <= p) j += step;
            }
            const long long oj = __shfl_sync(kAll, o, j);
            const int bx = __shfl_sync(kAll, box.x, j), by = __shfl_sync(kAll, box.y, j),
                      bz = __shfl_sync(kAll, box.z, j);
            const float r1 = __shfl_sync(kAll, rcp1, j), r2 = __shfl_sync(kAll, rcp2, j);
            if (p < wend) {
                const int32_t t = box_tile_small(s, bx, by, bz, r1, r2, int32_t(p - oj));
                atomicAdd(&row[t >> 2], 1u << ((t & 3) * 8));
            }
        }
    }
    __syncthreads();
    // tile t's byte is byte t of its row (little-endian words), so rows of words * 4 bytes
    uint32_t* dst = reinterpret_cast<uint32_t*>(cs_mat + bid * kCsRowsPerBlock * cs_mstride(ntiles));
    for (int i = threadIdx.x; i < kCsRowsPerBlock * words; i += kPrepThreads) dst[i] = cs_hist[i];
}

__global__ void __launch_bounds__(256) k_count_compat(const float* __restrict__ center,
                                                      const float* __restrict__ radius, int64_t n,
                                                      DevShape s, int4* __restrict__ boxes,
                                                      int64_t* __restrict__ counts, Status* status) {
    const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g == 0) counts[n] = 0;
    if (g >= n) return;
    float c[3] = {center[g * 3], center[g * 3 + 1], center[g * 3 + 2]};
    int4 box;
    int64_t cnt = tile_box(s, c, radius[g], &box);
    if (cnt <= 0) {
        atomicOr(&status->flags, GSV_FLAG_EMPTY_BOX);
        cnt = 0;
        box.w = 0;
    }
    boxes[g] = box;
    counts[g] = cnt;
}

// One thread per Gaussian writes its (tile, gid) pairs in raster order.
// One warp per 32 consecutive Gaussians.  Their pairs occupy one contiguous
// range of the output (offsets is an exclusive scan), which the lanes cover
// side by side: lane l writes pairs start+l, start+l+32, ... and finds the
// Gaussian a pair belongs to by a 5-step search over the warp's 32 offsets
// (coalesced, balanced however the pair counts are spread).  Tiles follow
// the (d,h,w) raster order of each Gaussian's tile box.
// Emission of the pairs in Gaussian-major (d,h,w) raster order
// (tile_voxelizer.py:126-145), plus the two fills the sort and the range
// pass need: the tile ranges cleared to (0,0) and the sort padding past the
// pair total (keys = ntiles, after every real tile) -- one launch.
// A warp owns 32 consecutive Gaussians and writes their pairs as one
// contiguous range: lane l takes pairs base + l, base + 32 + l, ... and finds
// its Gaussian by a shuffle binary search over the warp's first indices.
__global__ void __launch_bounds__(128) k_emit(const int4* __restrict__ boxes,
                                              const int64_t* __restrict__ offsets, int64_t n,
                                              DevShape s, int64_t cap, int32_t* __restrict__ keys,
                                              int32_t* __restrict__ vals, int2* __restrict__ ranges,
                                              int64_t ntiles, Status* status) {
    constexpr unsigned kAll = 0xffffffffu;
    const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int64_t total = offsets[n];
    if (g == 0) {
        if (total > cap) atomicOr(&status->flags, GSV_FLAG_CAPACITY_OVERFLOW);
        if (total > int64_t(INT32_MAX)) atomicOr(&status->flags, GSV_FLAG_TOO_MANY_PAIRS);
    }
    for (int64_t t = g; t < ntiles; t += stride) ranges[t] = make_int2(0, 0);
    for (int64_t i = total + g; i < cap; i += stride) {
        keys[i] = int32_t(ntiles);
        vals[i] = 0;
    }
    const int64_t g0 = g - lane;  // first Gaussian of this warp (warp-uniform)
    if (g0 >= n) return;
    const int m = int(min(int64_t(32), n - g0));
    const long long end = offsets[g0 + m];  // one past the warp's last pair
    int4 b = make_int4(0, 0, 0, 0);
    long long o = end;                      // lanes past the last Gaussian never match
    if (lane < m) {
        b = boxes[g];
        o = offsets[g];
    }
    const long long start = __shfl_sync(kAll, o, 0);
    for (long long base = start; base < end; base += 32) {
        const long long p = base + lane;
        int j = 0;  // largest j with o_j <= p
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
            const long long oj = __shfl_sync(kAll, o, j + step);
            if (oj <= p) j += step;
        }
        const long long oj = __shfl_sync(kAll, o, j);
        const int bx = __shfl_sync(kAll, b.x, j), by = __shfl_sync(kAll, b.y, j), bz = __shfl_sync(kAll, b.z, j);
        if (p >= end || p >= cap) continue;
        const int32_t c = int32_t(p - oj);
        const int32_t t0 = bx & 0xffff, t1 = (bx >> 16) & 0xffff, t2 = by & 0xffff;
        const int32_t n1 = bz & 0xffff, n2 = (bz >> 16) & 0xffff;
        const int32_t k = c % n2, r = c / n2;
        const int32_t jj = r % n1, i = r / n1;
        keys[p] = ((t0 + i) * s.nt[1] + (t1 + jj)) * s.nt[2] + (t2 + k);
        vals[p] = int32_t(g0 + j);
    }
}

// Tile ranges from the sorted keys; empty tiles stay (0,0).
__global__ void k_ranges(const int32_t* __restrict__ keys, const int64_t* __restrict__ offsets,
                         int64_t n, int64_t cap, int64_t ntiles, int2* __restrict__ ranges) {
    const int64_t total = min(offsets[n], cap);
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int32_t key = keys[i];
    if (key < 0 || key >= ntiles) return;
    if (i == 0 || keys[i - 1] != key) ranges[key].x = int32_t(i);
    if (i == total - 1 || keys[i + 1] != key) ranges[key].y = int32_t(i + 1);
}

// Column pass of the counting sort: one block per kCsCols tiles (dynamic
// block id from Status::pad[2]), 32 row groups per column.  cs_pos[r][t] =
// start(t) + the pairs of rows < r in tile t, where start(t) = the pairs in
// tiles < t, from a single-pass look-back over the blocks' tile totals.
// Writes every tile's range, (0,0) for an empty tile, clamped to `cap` (so a
// truncated list never reaches past the pair buffer).
__global__ void __launch_bounds__(kCsCols * kCsRowGroups) k_colscan(const uint8_t* __restrict__ mat,
                                                                    int32_t* __restrict__ pos, int64_t rows,
                                                                    int32_t ntiles, int64_t cap,
                                                                    int2* __restrict__ ranges, Status* status,
                                                                    unsigned long long* lb) {
    __shared__ int bid_s;
    __shared__ int64_t part[kCsRowGroups][kCsCols];  // a row group's sum, then its exclusive prefix
    __shared__ int64_t start_s[kCsCols], tot_s[kCsCols];
    if (threadIdx.x == 0) bid_s = atomicAdd(&status->pad[2], 1);
    __syncthreads();
    const int64_t bid = bid_s;
    const int c = threadIdx.x % kCsCols, rg = threadIdx.x / kCsCols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t = bid * kCsCols + c;
    const bool col_ok = t < ntiles;
    const int64_t per = (rows + kCsRowGroups - 1) / kCsRowGroups;
    const int64_t r0 = min(rows, rg * per), r1 = min(rows, r0 + per);
    int64_t sum = 0;
    if (col_ok) {
#pragma unroll 8
        for (int64_t r = r0; r < r1; ++r) sum += mat[r * cs_mstride(ntiles) + t];
    }
    part[rg][c] = sum;
    __syncthreads();
    if (warp == 0) {  // lane = column of this block
        int64_t run = 0;
        for (int k = 0; k < kCsRowGroups; ++k) {
            const int64_t v = part[k][lane];
            part[k][lane] = run;
            run += v;
        }
        tot_s[lane] = run;
        int64_t incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int64_t block_tot = __shfl_sync(0xffffffffu, incl, 31);
        const int64_t base = lookback(lb, bid, block_tot, status, lane);
        start_s[lane] = base + incl - run;
    }
    __syncthreads();
    if (!col_ok) return;
    int64_t at_r = start_s[c] + part[rg][c];
    for (int64_t r = r0; r < r1; ++r) {
        pos[r * ntiles + t] = int32_t(min(at_r, cap));
        at_r += mat[r * cs_mstride(ntiles) + t];
    }
    if (rg == 0) {
        const int64_t st = start_s[c], tt = tot_s[c];
        ranges[t] = tt > 0 ? make_int2(int32_t(min(st, cap)), int32_t(min(st + tt, cap))) : make_int2(0, 0);
    }
}

// Placement pass of the counting sort: one warp per row of kCsSeg
// Gaussians, kCsRowsPerBlock rows per block.  The warp copies its row of
// positions to shared memory, then walks the row's Gaussians in ascending
// id: the lanes take the Gaussian's tiles (distinct tiles, so no two lanes
// share a counter), write its id at each tile's current position and advance
// it.  Positions at or past `cap` are dropped (the overflow flag says so).
// Block 0 also latches the capacity flags and clears k_colscan's ticket
// counter and look-back words (k_colscan has finished: stream order).
__global__ void __launch_bounds__(32 * kCsRowsPerBlock) k_scatter(const int32_t* __restrict__ pos_in,
                                                                  const int4* __restrict__ boxes,
                                                                  const int64_t* __restrict__ offsets, int64_t n,
                                                                  int32_t ntiles, int64_t rows, DevShape s,
                                                                  int64_t cap, int32_t* __restrict__ pair_ids,
                                                                  Status* status, unsigned long long* lb,
                                                                  int64_t lb_words) {
    constexpr unsigned kAll = 0xffffffffu;
    extern __shared__ int32_t cs_at[];  // [kCsRowsPerBlock][ntiles]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            const int64_t total = offsets[n];
            if (total > cap) atomicOr(&status->flags, GSV_FLAG_CAPACITY_OVERFLOW);
            if (total > int64_t(INT32_MAX)) atomicOr(&status->flags, GSV_FLAG_TOO_MANY_PAIRS);
            status->pad[2] = 0;
        }
        for (int64_t i = threadIdx.x; i < lb_words; i += blockDim.x) lb[i] = 0ull;
    }
    const int64_t row = int64_t(blockIdx.x) * kCsRowsPerBlock + warp;
    if (row >= rows) return;  // warp-uniform; no block barrier follows
    int32_t* at_t = cs_at + warp * ntiles;
    for (int t = lane; t < ntiles; t += 32) at_t[t] = pos_in[row * ntiles + t];
    __syncwarp();
    const int64_t g0 = row * kCsSeg;
    for (int h = 0; h < kCsSeg; h += 32) {
        const int64_t gl = g0 + h + lane;
        const int4 mb = gl < n ? boxes[gl] : make_int4(0, 0, 0, 0);
        for (int k = 0; k < 32; ++k) {  // the Gaussians in ascending id
            const int cnt = __shfl_sync(kAll, mb.w, k);
            const int bx = __shfl_sync(kAll, mb.x, k), by = __shfl_sync(kAll, mb.y, k),
                      bz = __shfl_sync(kAll, mb.z, k);
            if (cnt <= 0) continue;  // warp-uniform
            const int32_t gid = int32_t(g0 + h + k);
            const float r1 = box_rcp(bz), r2 = box_rcp(bz >> 16);
            for (int c = lane; c < cnt; c += 32) {
                const int32_t t = box_tile_small(s, bx, by, bz, r1, r2, c);
                const int32_t p = at_t[t];
                if (p < cap) pair_ids[p] = gid;
                at_t[t] = int32_t(min(int64_t(p) + 1, cap));
            }
            __syncwarp();
        }
    }
}

int grid_for(int64_t items, int block) {
    int64_t g = (items + block - 1) / block;
    if (g < 1) g = 1;
    if (g > (int64_t(1) << 30)) g = int64_t(1) << 30;
    return int(g);
}

int sync_total(const GaussLayout& L, void* ws, int64_t n, int64_t* total_host, cudaStream_t st) {
    int64_t total = 0;
    GSV_CUDA_TRY(cudaMemcpyAsync(&total, at<int64_t>(ws, L.offsets) + n, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, st));
    GSV_CUDA_TRY(cudaStreamSynchronize(st));
    *total_host = total;
    return GSV_OK;
}

// Dynamic shared memory of k_prepare's byte counters and of k_scatter's positions.  Neither
// kernel declares static shared memory beyond a few words, and both stay within the 48 KB a
// launch may use without a function attribute.
int cs_prep_smem_bytes(int64_t ntiles) { return int(kCsRowsPerBlock * ((ntiles + 3) / 4) * int64_t(sizeof(uint32_t))); }
int cs_scatter_smem_bytes(int64_t ntiles) { return int(kCsRowsPerBlock * ntiles * int64_t(sizeof(int32_t))); }
static_assert(kCsRowsPerBlock * kCsMaxTiles * 4 <= 48 * 1024, "k_scatter's positions exceed 48 KB");
static_assert(kCsRowsPerBlock * kCsMaxTiles <= 40 * 1024, "k_prepare's counters leave no room for its static words");

// Shared tail of both binning flavours.  Counting sort (k_colscan,
// k_scatter) when the preprocess wrote the per-row tile counts (native path,
// small tile count) and `mode` allows it; otherwise emit, radix sort, ranges.
int bin_common(const ShapeInfo& si, int64_t n, void* ws_gauss, void* ws_pairs, size_t ws_pairs_bytes,
               int64_t cap, int32_t* vals_out_override, int mode, bool rows_written, cudaStream_t st) {
    if (cap < 0 || cap > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    if (mode != GSV_BIN_AUTO && mode != GSV_BIN_RADIX && mode != GSV_BIN_COUNTING) return GSV_ERR_INVALID_ARGUMENT;
    const GaussLayout G = gauss_layout(n, si);
    const PairLayout P = pair_layout(cap, si, 0);
    if (ws_pairs_bytes < P.total || !ws_pairs) return GSV_ERR_INVALID_ARGUMENT;
    DevShape s = dev_shape(si);
    Status* status = at<Status>(ws_gauss, G.status);
    const int64_t* offsets = at<int64_t>(ws_gauss, G.offsets);
    int32_t* keys_in = at<int32_t>(ws_pairs, P.keys_in);
    int32_t* vals_in = at<int32_t>(ws_pairs, P.vals_in);
    int32_t* keys_out = at<int32_t>(ws_pairs, P.keys_out);
    int32_t* vals_out = vals_out_override ? vals_out_override : at<int32_t>(ws_pairs, P.vals_out);
    int2* ranges = at<int2>(ws_gauss, G.ranges);
    const bool cs = rows_written && G.cs;
    if (mode == GSV_BIN_COUNTING && !cs) return GSV_ERR_INVALID_ARGUMENT;
    if (cap == 0) {
        GSV_CUDA_TRY(cudaMemsetAsync(ranges, 0, size_t(si.ntiles) * sizeof(int2), st));
        return GSV_OK;
    }
    if (cs && mode != GSV_BIN_RADIX) {
        unsigned long long* lb_cs = reinterpret_cast<unsigned long long*>(status + 1) + prep_blocks(n);
        const int64_t rows = cs_rows(n);
        const int32_t T = int32_t(si.ntiles);
        k_colscan<<<unsigned(cs_col_blocks(T)), kCsCols * kCsRowGroups, 0, st>>>(
            at<uint8_t>(ws_gauss, G.cs_mat), at<int32_t>(ws_gauss, G.cs_pos), rows, T, cap, ranges, status, lb_cs);
        GSV_LAUNCH_CHECK();
        const int smem = cs_scatter_smem_bytes(T);
        k_scatter<<<unsigned(prep_blocks(n)), 32 * kCsRowsPerBlock, smem, st>>>(
            at<int32_t>(ws_gauss, G.cs_pos), at<int4>(ws_gauss, G.box), offsets, n, T, rows, s, cap, vals_out, status,
            lb_cs, cs_col_blocks(T));
        GSV_LAUNCH_CHECK();
        return GSV_OK;
    }
    // enough CTAs for the emission (one thread per Gaussian) and for the fills
    const int fill_grid = grid_for(cap > si.ntiles ? cap : si.ntiles, 128);
    const int emit_grid = grid_for(n, 128);
    const int grid = emit_grid > (fill_grid < 1184 ? fill_grid : 1184) ? emit_grid : (fill_grid < 1184 ? fill_grid : 1184);
    k_emit<<<grid, 128, 0, st>>>(at<int4>(ws_gauss, G.box), offsets, n, s, cap, keys_in, vals_in, ranges,
                                 si.ntiles, status);
    GSV_LAUNCH_CHECK();
    size_t sort_bytes = P.sort_tmp_bytes;
    GSV_CUDA_TRY(cub::DeviceRadixSort::SortPairs(at<void>(ws_pairs, P.sort_tmp), sort_bytes, keys_in,
                                                 keys_out, vals_in, vals_out, int(cap), 0,
                                                 sort_end_bit(si.ntiles), st));
    k_ranges<<<grid_for(cap, 256), 256, 0, st>>>(keys_out, offsets, n, cap, si.ntiles, ranges);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points
// ---------------------------------------------------------------------------

void gsv_detail_set_error(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "%s (%s) at %s:%d: %s", cudaGetErrorName(e), what,
             file, line, cudaGetErrorString(e));
}

extern "C" {

const char* gsv_last_error(void) { return g_last_error; }

int gsv_abi_version(void) { return GSV_ABI_VERSION; }

const char* gsv_status_string(int status) {
    switch (status) {
        case GSV_OK: return "ok";
        case GSV_ERR_INVALID_ARGUMENT: return "invalid argument";
        case GSV_ERR_CAPACITY: return "pair capacity exceeded";
        case GSV_ERR_CUDA: return "CUDA error";
        case GSV_ERR_EMPTY_BOX: return "empty tile box (negative radius)";
        case GSV_ERR_TOO_MANY_PAIRS: return "more than INT32_MAX tile pairs";
        default: return "unknown status";
    }
}

int64_t gsv_num_tiles(gsv_shape shape) {
    ShapeInfo si = shape_info(shape);
    return si.ok ? si.ntiles : -1;
}

size_t gsv_gauss_workspace_bytes(int64_t n, gsv_shape shape) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || n >= int64_t(INT32_MAX)) return 0;
    return gauss_layout(n, si).total;
}

size_t gsv_pair_workspace_bytes(int64_t capacity, gsv_shape shape, int flags) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || capacity < 0 || capacity > int64_t(INT32_MAX)) return 0;
    return pair_layout(capacity, si, flags).total;
}

static int prepare_impl(const gsv_params* p, const int32_t* live, gsv_shape shape, void* ws_gauss,
                        size_t ws_gauss_bytes, int64_t* total_pairs_host, void* stream) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || !p || p->n < 0 || p->n >= int64_t(INT32_MAX) || !ws_gauss) return GSV_ERR_INVALID_ARGUMENT;
    const int64_t n = p->n;
    if (n > 0 && (!p->positions || !p->scales || !p->rotations || !p->density_r || !p->density_i))
        return GSV_ERR_INVALID_ARGUMENT;
    const GaussLayout L = gauss_layout(n, si);
    if (ws_gauss_bytes < L.total) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Status* status = at<Status>(ws_gauss, L.status);
    // status flags, the block counters and the scans' look-back words
    GSV_CUDA_TRY(cudaMemsetAsync(status, 0, status_bytes(n, si.ntiles), st));
    const int smem = L.cs ? cs_prep_smem_bytes(si.ntiles) : 0;
    k_prepare<<<unsigned(prep_blocks(n)), kPrepThreads, smem, st>>>(
        p->positions, p->scales, p->rotations, p->density_r, p->density_i, n, live, dev_shape(si),
        at<Rec>(ws_gauss, L.rec), at<float4>(ws_gauss, L.ext), at<int4>(ws_gauss, L.box),
        at<int64_t>(ws_gauss, L.offsets), status, L.cs ? at<uint8_t>(ws_gauss, L.cs_mat) : nullptr,
        int32_t(si.ntiles), at<float>(ws_gauss, L.accum));
    GSV_LAUNCH_CHECK();
    if (total_pairs_host) return sync_total(L, ws_gauss, n, total_pairs_host, st);
    return GSV_OK;
}

int gsv_prepare(const gsv_params* p, gsv_shape shape, void* ws_gauss, size_t ws_gauss_bytes,
                int64_t* total_pairs_host, void* stream) {
    return prepare_impl(p, nullptr, shape, ws_gauss, ws_gauss_bytes, total_pairs_host, stream);
}

int gsv_prepare_live(const gsv_params* p, const int32_t* live, gsv_shape shape, void* ws_gauss,
                     size_t ws_gauss_bytes, int64_t* total_pairs_host, void* stream) {
    if (!live) return GSV_ERR_INVALID_ARGUMENT;
    return prepare_impl(p, live, shape, ws_gauss, ws_gauss_bytes, total_pairs_host, stream);
}

int gsv_bin_ex(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, size_t ws_pairs_bytes,
               int64_t capacity, int mode, void* stream) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || !ws_gauss) return GSV_ERR_INVALID_ARGUMENT;
    return bin_common(si, n, ws_gauss, ws_pairs, ws_pairs_bytes, capacity, nullptr, mode, true,
                      static_cast<cudaStream_t>(stream));
}

int gsv_bin(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, size_t ws_pairs_bytes,
            int64_t capacity, void* stream) {
    return gsv_bin_ex(shape, n, ws_gauss, ws_pairs, ws_pairs_bytes, capacity, GSV_BIN_AUTO, stream);
}

int gsv_bin_views(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs, int64_t capacity,
                  int32_t** tile_ranges, int32_t** pair_ids) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || !ws_gauss || !ws_pairs) return GSV_ERR_INVALID_ARGUMENT;
    if (tile_ranges) *tile_ranges = at<int32_t>(ws_gauss, gauss_layout(n, si).ranges);
    if (pair_ids) *pair_ids = at<int32_t>(ws_pairs, pair_layout(capacity, si, 0).vals_out);
    return GSV_OK;
}

int gsv_status_views(gsv_shape shape, int64_t n, void* ws_gauss, int32_t** flags, int64_t** total_pairs) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || !ws_gauss) return GSV_ERR_INVALID_ARGUMENT;
    const GaussLayout L = gauss_layout(n, si);
    if (flags) *flags = &at<Status>(ws_gauss, L.status)->flags;
    if (total_pairs) *total_pairs = at<int64_t>(ws_gauss, L.offsets) + n;
    return GSV_OK;
}

int gsv_read_status(gsv_shape shape, int64_t n, const void* ws_gauss, int64_t* total_pairs,
                    int32_t* flags, void* stream) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || !ws_gauss) return GSV_ERR_INVALID_ARGUMENT;
    const GaussLayout L = gauss_layout(n, si);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t total = 0;
    Status s{};
    GSV_CUDA_TRY(cudaMemcpyAsync(&total, at<int64_t>(ws_gauss, L.offsets) + n, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, st));
    GSV_CUDA_TRY(cudaMemcpyAsync(&s, at<Status>(ws_gauss, L.status), sizeof(Status),
                                 cudaMemcpyDeviceToHost, st));
    GSV_CUDA_TRY(cudaStreamSynchronize(st));
    if (total_pairs) *total_pairs = total;
    if (flags) *flags = s.flags;
    return GSV_OK;
}

int gsv_build_tile_pairs_count(const float* center_vox, const float* radius_vox, int64_t n,
                               gsv_shape shape, void* ws_gauss, size_t ws_gauss_bytes,
                               int64_t* total_pairs_host, void* stream) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || n >= int64_t(INT32_MAX) || !ws_gauss) return GSV_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!center_vox || !radius_vox)) return GSV_ERR_INVALID_ARGUMENT;
    const GaussLayout L = gauss_layout(n, si);
    if (ws_gauss_bytes < L.total) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Status* status = at<Status>(ws_gauss, L.status);
    GSV_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(Status), st));
    k_count_compat<<<grid_for(n + 1, 256), 256, 0, st>>>(center_vox, radius_vox, n, dev_shape(si),
                                                         at<int4>(ws_gauss, L.box),
                                                         at<int64_t>(ws_gauss, L.counts), status);
    GSV_LAUNCH_CHECK();
    size_t scan_bytes = L.scan_tmp_bytes;
    GSV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(at<void>(ws_gauss, L.scan_tmp), scan_bytes,
                                               at<int64_t>(ws_gauss, L.counts),
                                               at<int64_t>(ws_gauss, L.offsets), int(n + 1), st));
    if (total_pairs_host) return sync_total(L, ws_gauss, n, total_pairs_host, st);
    return GSV_OK;
}

int gsv_build_tile_pairs_fill(gsv_shape shape, int64_t n, void* ws_gauss, void* ws_pairs,
                              size_t ws_pairs_bytes, int64_t capacity, int32_t* tile_ranges,
                              int32_t* pair_ids, void* stream) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0 || !ws_gauss || !tile_ranges || (capacity > 0 && !pair_ids))
        return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = bin_common(si, n, ws_gauss, ws_pairs, ws_pairs_bytes, capacity, pair_ids, GSV_BIN_RADIX, false, st);
    if (rc != GSV_OK) return rc;
    const GaussLayout L = gauss_layout(n, si);
    GSV_CUDA_TRY(cudaMemcpyAsync(tile_ranges, at<int2>(ws_gauss, L.ranges), size_t(si.ntiles) * sizeof(int2),
                                 cudaMemcpyDeviceToDevice, st));
    return GSV_OK;
}

}  // extern "C"

// Internal accessors for the render translation unit.
namespace gsv {
int layout_for(gsv_shape shape, int64_t n, int64_t cap, int flags, GaussLayout* G, PairLayout* P,
               int64_t* ntiles) {
    ShapeInfo si = shape_info(shape);
    if (!si.ok || n < 0) return GSV_ERR_INVALID_ARGUMENT;
    if (G) *G = gauss_layout(n, si);
    if (P) *P = pair_layout(cap, si, flags);
    if (ntiles) *ntiles = si.ntiles;
    return GSV_OK;
}
}  // namespace gsv
