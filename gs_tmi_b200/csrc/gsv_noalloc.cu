// gsv_noalloc.cu -- tile binning that allocates no device memory.
//
// Some callers cannot allocate device memory at all: their GPU memory is
// owned by another allocator (a framework that reserves the device up front,
// a process with a hard memory cap), or they run on a path with a fixed
// memory plan where no allocation may happen.  For them this file offers
// gsv_build_tile_pairs_noalloc: the same result as
// gsv_build_tile_pairs_count + gsv_build_tile_pairs_fill, with every scratch
// buffer (tile boxes, counts, offsets, sort keys, sort temporaries) carved
// from one file-scope __device__ array instead of a caller workspace.
//
// The array is kNoallocScratchBytes (40 MiB + the CUB temporaries), is
// created on every GPU that loads this code and stays there until the
// process exits.  Sizes: at most kMaxGaussians Gaussians and kMaxPairs
// (tile, Gaussian) pairs per call.
//
// In host code the array's name is only a host-side stand-in, never a device
// address.  The first call on each device (with that device current) looks
// up the real address with cudaGetSymbolAddress and caches it.  The call
// synchronises its stream once (to read the pair total back).  All calls
// share the one array and it keeps the previous call's contents: the entry
// point clears what must start at zero, and calls that overlap on the GPU
// (two streams or threads at once) race on it, so callers must serialise
// them.
#include <cub/cub.cuh>

#include <mutex>

#include "gsv_common.cuh"

using namespace gsv;

namespace {

constexpr int64_t kMaxGaussians = int64_t(1) << 18;  // 262,144
constexpr int64_t kMaxPairs = int64_t(1) << 21;      // 2,097,152
constexpr int kMaxTilesPerAxisNA = 65535;
constexpr size_t kSortTmpReserve = size_t(8) << 20;  // checked against CUB at set-up
constexpr size_t kScanTmpReserve = size_t(1) << 20;

constexpr size_t al(size_t x) { return (x + 255) & ~size_t(255); }

// Layout of the scratch array (byte offsets).
constexpr size_t kOffBoxes = 0;
constexpr size_t kOffCounts = al(kOffBoxes + size_t(kMaxGaussians) * sizeof(int4));
constexpr size_t kOffOffsets = al(kOffCounts + size_t(kMaxGaussians + 1) * sizeof(int64_t));
constexpr size_t kOffScanTmp = al(kOffOffsets + size_t(kMaxGaussians + 1) * sizeof(int64_t));
constexpr size_t kOffStatus = al(kOffScanTmp + kScanTmpReserve);
constexpr size_t kOffKeysIn = al(kOffStatus + 256);
constexpr size_t kOffValsIn = al(kOffKeysIn + size_t(kMaxPairs) * sizeof(int32_t));
constexpr size_t kOffKeysOut = al(kOffValsIn + size_t(kMaxPairs) * sizeof(int32_t));
constexpr size_t kOffSortTmp = al(kOffKeysOut + size_t(kMaxPairs) * sizeof(int32_t));
constexpr size_t kNoallocScratchBytes = al(kOffSortTmp + kSortTmpReserve);

// The scratch itself.  Host code must not use this name as a pointer.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_dev[kMaxDevices] = {nullptr};

struct NaShape {
    int32_t size[3];
    int32_t nt[3];
    int32_t ts;
    int64_t ntiles;
};

__global__ void __launch_bounds__(256) k_na_count(const float* __restrict__ center,
                                                  const float* __restrict__ radius, int64_t n, NaShape s,
                                                  int4* __restrict__ boxes, int64_t* __restrict__ counts,
                                                  int32_t* __restrict__ flags) {
    const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g == 0) counts[n] = 0;
    if (g >= n) return;
    int32_t tlo[3], na[3];
    int64_t cnt = 1;
    const float r = radius[g];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float c = center[g * 3 + a];
        // floor/ceil of center -/+ radius, clamp, // tile, clamp (tile_voxelizer.py:97-114)
        int32_t lo = __float2int_rz(floorf(__fsub_rn(c, r)));
        int32_t hi = __float2int_rz(ceilf(__fadd_rn(c, r)));
        lo = min(max(lo, 0), s.size[a] - 1);
        hi = min(max(hi, 0), s.size[a] - 1);
        const int32_t t0 = min(max(lo / s.ts, 0), s.nt[a] - 1);
        const int32_t t1 = min(max(hi / s.ts, 0), s.nt[a] - 1);
        tlo[a] = t0;
        na[a] = t1 - t0 + 1;
        if (na[a] <= 0) cnt = 0;
        else cnt *= na[a];
    }
    if (cnt <= 0) {
        atomicOr(flags, GSV_FLAG_EMPTY_BOX);
        cnt = 0;
    }
    boxes[g] = make_int4(tlo[0] | (tlo[1] << 16), tlo[2] | (max(na[0], 0) << 16),
                         max(na[1], 0) | (max(na[2], 0) << 16), int32_t(cnt));
    counts[g] = cnt;
}

// Pairs in Gaussian-major (d,h,w) raster order (tile_voxelizer.py:126-145).
// A warp owns 32 consecutive Gaussians and writes their pairs as one
// contiguous range: lane l takes pairs base + l, base + 32 + l, ... and finds
// its Gaussian by a shuffle binary search over the warp's first indices, so
// one large Gaussian is spread over the warp and the stores are coalesced.
__global__ void __launch_bounds__(128) k_na_emit(const int4* __restrict__ boxes,
                                                 const int64_t* __restrict__ offsets, int64_t n, NaShape s,
                                                 int32_t* __restrict__ keys, int32_t* __restrict__ vals) {
    constexpr unsigned kAll = 0xffffffffu;
    const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int64_t g0 = g - lane;  // first Gaussian of this warp (warp-uniform)
    if (g0 >= n) return;
    const int m = int(min(int64_t(32), n - g0));
    const long long end = offsets[g0 + m];  // one past the warp's last pair
    int4 b = make_int4(0, 0, 0, 0);
    long long o = end;  // lanes past the last Gaussian never match
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
        if (p >= end) continue;
        const int32_t c = int32_t(p - oj);
        const int32_t t0 = bx & 0xffff, t1 = (bx >> 16) & 0xffff, t2 = by & 0xffff;
        const int32_t n1 = bz & 0xffff, n2 = (bz >> 16) & 0xffff;
        const int32_t k = c % n2, r = c / n2;
        const int32_t jj = r % n1, i = r / n1;
        keys[p] = ((t0 + i) * s.nt[1] + (t1 + jj)) * s.nt[2] + (t2 + k);
        vals[p] = int32_t(g0 + j);
    }
}

__global__ void k_na_ranges(const int32_t* __restrict__ keys, int64_t total, int2* __restrict__ ranges) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int32_t key = keys[i];
    if (i == 0 || keys[i - 1] != key) ranges[key].x = int32_t(i);
    if (i == total - 1 || keys[i + 1] != key) ranges[key].y = int32_t(i + 1);
}

int na_end_bit(int64_t ntiles) {
    int bits = 1;
    while ((int64_t(1) << bits) <= ntiles) ++bits;
    return bits;
}

// Once per device: the device address of the scratch array, and a check that
// the CUB temporaries for the largest allowed problem fit their reserves.
int na_scratch(void** out) {
    int dev = 0;
    GSV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return GSV_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        size_t scan_bytes = 0, sort_bytes = 0;
        GSV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int64_t*)nullptr,
                                                   (int64_t*)nullptr, int(kMaxGaussians + 1)));
        cub::DoubleBuffer<int32_t> k(nullptr, nullptr), v(nullptr, nullptr);
        GSV_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k, v, int(kMaxPairs), 0, 31));
        if (scan_bytes > kScanTmpReserve || sort_bytes > kSortTmpReserve) return GSV_ERR_INVALID_ARGUMENT;
        void* p = nullptr;
        GSV_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_dev[dev] = p;
    }
    *out = g_scratch_dev[dev];
    return GSV_OK;
}

}  // namespace

extern "C" int gsv_build_tile_pairs_noalloc(const float* center_vox, const float* radius_vox, int64_t n,
                                            gsv_shape shape, int32_t* tile_ranges, int32_t* pair_ids,
                                            int64_t pair_capacity, int64_t* total_pairs, void* stream) {
    if (shape.d <= 0 || shape.h <= 0 || shape.w <= 0 || shape.tile_size <= 0 || shape.d >= (1 << 24) ||
        shape.h >= (1 << 24) || shape.w >= (1 << 24))
        return GSV_ERR_INVALID_ARGUMENT;
    if (n < 0 || n > kMaxGaussians || !tile_ranges || !total_pairs || pair_capacity < 0 ||
        (n > 0 && (!center_vox || !radius_vox)))
        return GSV_ERR_INVALID_ARGUMENT;
    NaShape s{};
    s.size[0] = shape.d; s.size[1] = shape.h; s.size[2] = shape.w;
    s.ts = shape.tile_size;
    for (int a = 0; a < 3; ++a) {
        s.nt[a] = (s.size[a] + s.ts - 1) / s.ts;
        if (s.nt[a] > kMaxTilesPerAxisNA) return GSV_ERR_INVALID_ARGUMENT;
    }
    s.ntiles = int64_t(s.nt[0]) * s.nt[1] * s.nt[2];
    if (s.ntiles >= (int64_t(1) << 30)) return GSV_ERR_INVALID_ARGUMENT;

    void* base = nullptr;
    const int rc = na_scratch(&base);
    if (rc != GSV_OK) return rc;
    char* sc = static_cast<char*>(base);
    int4* boxes = reinterpret_cast<int4*>(sc + kOffBoxes);
    int64_t* counts = reinterpret_cast<int64_t*>(sc + kOffCounts);
    int64_t* offsets = reinterpret_cast<int64_t*>(sc + kOffOffsets);
    int32_t* flags = reinterpret_cast<int32_t*>(sc + kOffStatus);
    int32_t* keys_in = reinterpret_cast<int32_t*>(sc + kOffKeysIn);
    int32_t* vals_in = reinterpret_cast<int32_t*>(sc + kOffValsIn);
    int32_t* keys_out = reinterpret_cast<int32_t*>(sc + kOffKeysOut);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Part 1: boxes, counts, offsets, pair total (one host sync, as the
    // reference's .item() at tile_voxelizer.py:118).
    GSV_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int32_t), st));
    k_na_count<<<unsigned((n + 256) / 256), 256, 0, st>>>(center_vox, radius_vox, n, s, boxes, counts, flags);
    GSV_LAUNCH_CHECK();
    size_t scan_bytes = kScanTmpReserve;
    GSV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(sc + kOffScanTmp, scan_bytes, counts, offsets, int(n + 1), st));
    int64_t total = 0;
    int32_t fl = 0;
    GSV_CUDA_TRY(cudaMemcpyAsync(&total, offsets + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    GSV_CUDA_TRY(cudaMemcpyAsync(&fl, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GSV_CUDA_TRY(cudaStreamSynchronize(st));
    *total_pairs = total;
    if (fl & GSV_FLAG_EMPTY_BOX) return GSV_ERR_EMPTY_BOX;
    if (total > kMaxPairs || total > pair_capacity) return GSV_ERR_CAPACITY;

    // Part 2: pairs, stable radix sort by tile, ranges (empty tiles (0,0)).
    GSV_CUDA_TRY(cudaMemsetAsync(tile_ranges, 0, size_t(s.ntiles) * sizeof(int2), st));
    if (total == 0) return GSV_OK;
    if (!pair_ids) return GSV_ERR_INVALID_ARGUMENT;
    k_na_emit<<<unsigned((n + 127) / 128), 128, 0, st>>>(boxes, offsets, n, s, keys_in, vals_in);
    GSV_LAUNCH_CHECK();
    // ping-pong between scratch and the caller's pair_ids (no internal copies)
    cub::DoubleBuffer<int32_t> dk(keys_in, keys_out), dv(vals_in, pair_ids);
    size_t sort_bytes = kSortTmpReserve;
    GSV_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sc + kOffSortTmp, sort_bytes, dk, dv, int(total), 0,
                                                 na_end_bit(s.ntiles), st));
    if (dv.Current() != pair_ids)
        GSV_CUDA_TRY(cudaMemcpyAsync(pair_ids, dv.Current(), size_t(total) * sizeof(int32_t),
                                     cudaMemcpyDeviceToDevice, st));
    k_na_ranges<<<unsigned((total + 255) / 256), 256, 0, st>>>(dk.Current(), total,
                                                               reinterpret_cast<int2*>(tile_ranges));
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}
