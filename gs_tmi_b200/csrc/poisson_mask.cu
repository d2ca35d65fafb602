// poisson_mask.cu -- variable-density Poisson-disc k-space masks, a batch per
// launch, one CTA per mask.
//
// Reference: 3DGS/3dgsVC/data/mask_generator.py:241-390
// (_generate_poisson_mask_heuristic).  After the calibration square is set,
// the pixels are visited once in a random order; a pixel is taken unless it
// is set already or a taken pixel p lies at |p - c|^2 < r(c)^2, and the pass
// stops once `target` pixels are set.  That pass is sequential: whether c is
// taken depends on every earlier decision in its disc.
//
// Here the pass is an order-respecting parallel greedy.  With q(c) the
// position of c in the visiting order, an undecided pixel c is
//   rejected  as soon as its disc holds a calibration pixel or a taken p
//             with q(p) < q(c) (that p is set when the sequential pass
//             reaches c, whatever happens in between), and
//   taken     once no p in its disc with q(p) < q(c) is undecided and none
//             is taken (then nothing set before c lies in its disc);
// otherwise it waits for the next round.  Decisions never change, so each
// one equals the sequential pass's, and the lowest undecided pixel always
// decides: the rounds end (about ten for 256x256).  The pass's stop at
// `target` keeps the first target - |calibration| taken pixels in visiting
// order, found with one block-wide scan.  Threads take the pixels in visiting
// order (thread t: positions t, t + 1024, ...) and read decisions made in the
// same round, which shortens the chains.  The per-pixel state lives in shared
// memory (1 byte per pixel); the visiting positions in a global workspace.
#include <cub/cub.cuh>

#include "gsv_common.cuh"

namespace {

constexpr int kThreads = 1024;
constexpr int kMaxPixels = 196608;  // state bytes in shared memory (192 KB)

enum : int8_t { kUndecided = 0, kTaken = 1, kRejected = 2, kCalib = 3 };

// Python slice bounds [lo, hi) of start:stop on an axis of size n.
__host__ __device__ inline void py_slice(int start, int stop, int n, int* lo, int* hi) {
    if (start < 0) start += n;
    if (stop < 0) stop += n;
    start = start < 0 ? 0 : (start > n ? n : start);
    stop = stop < 0 ? 0 : (stop > n ? n : stop);
    *lo = start;
    *hi = stop > start ? stop : start;
}

// Decision for pixel c at visiting position q.
__device__ int8_t decide(int c, int q, int ny, int nz, const double* __restrict__ radius,
                         const int32_t* __restrict__ pos, const int8_t* st) {
    const int y = c / nz, z = c - (c / nz) * nz;
    const double r = radius[c];
    const double r2 = r * r;
    // ceil(r), bounded by the plane (a larger window holds no more pixels)
    const int ir = (r > 0.0) ? int(fmin(ceil(r), double(max(ny, nz)))) : 0;
    bool wait = false;
    // rows and columns centre-out: near pixels first, so a rejection is found early
    for (int a = 0; a <= 2 * ir; ++a) {
        const int dy = (a & 1) ? -((a + 1) >> 1) : (a >> 1);
        const int py = y + dy;
        if (py < 0 || py >= ny) continue;
        const double dy2 = double(dy) * dy;
        if (!(dy2 < r2)) continue;
        for (int b = 0; b <= 2 * ir; ++b) {
            const int dz = (b & 1) ? -((b + 1) >> 1) : (b >> 1);
            const double d2 = dy2 + double(dz) * dz;
            if (!(d2 < r2)) break;  // |dz| never shrinks along b (0, -1, +1, -2, +2, ...)
            const int pz = z + dz;
            if (pz < 0 || pz >= nz || (dy == 0 && dz == 0)) continue;
            const int p = py * nz + pz;
            const int8_t s = st[p];
            if (s == kRejected) continue;
            if (s == kCalib) return kRejected;
            if (s == kTaken) {
                if (pos[p] < q) return kRejected;
            } else if (!wait && pos[p] < q) {
                wait = true;
            }
        }
    }
    return wait ? kUndecided : kTaken;
}

__global__ void __launch_bounds__(kThreads, 1) k_poisson(const double* __restrict__ radius,
                                                         const int32_t* __restrict__ orders, int ny, int nz,
                                                         int calib, int64_t target, int8_t* __restrict__ masks,
                                                         int32_t* __restrict__ rounds_out,
                                                         int32_t* __restrict__ positions) {
    extern __shared__ int8_t st[];
    using Scan = cub::BlockScan<int, kThreads>;
    __shared__ typename Scan::TempStorage scan_tmp;
    const int n = ny * nz;
    const int64_t b = blockIdx.x;
    const int32_t* order = orders + b * n;
    int32_t* pos = positions + b * n;
    int8_t* out = masks + b * n;
    const int t = threadIdx.x;

    // visiting position of every pixel; the order must be a permutation
    for (int i = t; i < n; i += kThreads) pos[i] = -1;
    __syncthreads();
    bool bad = false;
    for (int q = t; q < n; q += kThreads) {
        const int c = order[q];
        if (c < 0 || c >= n) bad = true;
        else pos[c] = q;
    }
    __syncthreads();
    for (int i = t; i < n; i += kThreads) bad |= pos[i] < 0;
    bad = __syncthreads_or(bad);

    int y0, y1, z0, z1;
    py_slice(ny / 2 - calib / 2, ny / 2 + calib / 2, ny, &y0, &y1);
    py_slice(nz / 2 - calib / 2, nz / 2 + calib / 2, nz, &z0, &z1);
    const int64_t n_calib = int64_t(y1 - y0) * (z1 - z0);
    for (int i = t; i < n; i += kThreads) {
        const int y = i / nz, z = i - (i / nz) * nz;
        st[i] = (y >= y0 && y < y1 && z >= z0 && z < z1) ? kCalib : kUndecided;
    }
    __syncthreads();

    int rounds = 0;
    if (!bad && n_calib < target) {
        for (; rounds <= n; ++rounds) {  // the lowest undecided pixel decides every round
            bool left = false;
            for (int q = t; q < n; q += kThreads) {
                const int c = order[q];
                if (st[c] != kUndecided) continue;
                const int8_t d = decide(c, q, ny, nz, radius, pos, st);
                if (d == kUndecided) left = true;
                else st[c] = d;
            }
            if (!__syncthreads_or(left)) {
                ++rounds;
                break;
            }
        }
        // keep the first target - n_calib taken pixels in visiting order
        const int64_t keep = target - n_calib;
        const int chunk = (n + kThreads - 1) / kThreads;
        const int q0 = t * chunk, q1 = min(n, q0 + chunk);
        int mine = 0;
        for (int q = q0; q < q1; ++q) mine += st[order[q]] == kTaken;
        int before = 0;
        Scan(scan_tmp).ExclusiveSum(mine, before);
        int64_t idx = before;
        for (int q = q0; q < q1; ++q) {
            const int c = order[q];
            if (st[c] == kTaken) {
                if (idx >= keep) st[c] = kRejected;
                ++idx;
            }
        }
        __syncthreads();
    }
    for (int i = t; i < n; i += kThreads) out[i] = (st[i] == kTaken || st[i] == kCalib) ? 1 : 0;
    if (t == 0 && rounds_out) rounds_out[b] = bad ? -1 : rounds;
}

}  // namespace

extern "C" {

size_t gsv_poisson_workspace_bytes(int32_t ny, int32_t nz, int32_t count) {
    if (ny <= 0 || nz <= 0 || count <= 0 || int64_t(ny) * nz > kMaxPixels) return 0;
    return size_t(count) * size_t(ny) * size_t(nz) * sizeof(int32_t);
}

int gsv_poisson_masks(const double* radius, const int32_t* orders, int32_t ny, int32_t nz, int32_t calib,
                      int64_t target, int32_t count, int8_t* masks, int32_t* rounds, void* ws, size_t ws_bytes,
                      void* stream) {
    if (ny <= 0 || nz <= 0 || count < 0 || calib < 0 || int64_t(ny) * nz > kMaxPixels) return GSV_ERR_INVALID_ARGUMENT;
    if (count == 0) return GSV_OK;
    if (!radius || !orders || !masks || !ws || ws_bytes < gsv_poisson_workspace_bytes(ny, nz, count))
        return GSV_ERR_INVALID_ARGUMENT;
    const int smem = ny * nz;
    GSV_CUDA_TRY(cudaFuncSetAttribute(k_poisson, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_poisson<<<count, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(
        radius, orders, ny, nz, calib, target, masks, rounds, static_cast<int32_t*>(ws));
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
