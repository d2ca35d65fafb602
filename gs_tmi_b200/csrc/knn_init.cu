// knn_init.cu -- exact 3-nearest-neighbour distances of voxel-centred seeds,
// for the intensity-seeded scale initialisation of 3DGSMR
// (3DGS/3dgsVC/gaussian/gaussian_model.py:283-306, _sampled_3nn_scale_init:
// cKDTree on the normalised positions, mean distance to the 3 nearest other
// seeds, at least 1e-6, the last distance repeated when fewer than 3 exist,
// 1e-3 for a lone seed).
//
// The seeds are distinct voxels, so an occupancy grid replaces the k-d
// tree: each seed scans Chebyshev shells r = 1, 2, ... of voxels around its
// own and stops once the nearest possible point of the next shell,
// r * min_a(2 / shape_a) in normalised units (less a 1e-6 margin for the
// rounding of the FP32 positions), lies beyond its current third neighbour.
// Distances come from the caller's FP32 positions in FP64, then round to
// FP32, and the mean is taken in FP32 -- what the k-d tree query and the
// reference's float32 mean compute.
#include "gsv_common.cuh"

namespace {

constexpr int kBlock = 256;

__global__ void k_mark(const int64_t* __restrict__ vox, int64_t n, int32_t* __restrict__ grid) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        grid[vox[i]] = int32_t(i);
}

__device__ __forceinline__ void insert3(double d2, double best[3]) {
    if (d2 < best[2]) {
        if (d2 < best[1]) {
            best[2] = best[1];
            if (d2 < best[0]) {
                best[1] = best[0];
                best[0] = d2;
            } else {
                best[1] = d2;
            }
        } else {
            best[2] = d2;
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_knn3(const int64_t* __restrict__ vox, const float* __restrict__ pos,
                                                 int64_t n, int32_t d, int32_t h, int32_t w,
                                                 const int32_t* __restrict__ grid, float* __restrict__ out) {
    const double umin = 2.0 / double(max(d, max(h, w)));
    const int rmax = max(d, max(h, w));
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = vox[i];
        const int z = int(v / (int64_t(h) * w)), y = int((v / w) % h), x = int(v % w);
        const double p0 = pos[i * 3], p1 = pos[i * 3 + 1], p2 = pos[i * 3 + 2];
        double best[3] = {inf, inf, inf};
        for (int r = 1; r <= rmax; ++r) {
            const double lo = double(r) * umin - 1e-6;
            if (lo > 0.0 && lo * lo > best[2]) break;  // nothing on this shell or beyond can improve
            for (int dz = -r; dz <= r; ++dz) {
                const int zz = z + dz;
                if (zz < 0 || zz >= d) continue;
                for (int dy = -r; dy <= r; ++dy) {
                    const int yy = y + dy;
                    if (yy < 0 || yy >= h) continue;
                    const bool face = (dz == -r || dz == r || dy == -r || dy == r);
                    const int step = face ? 1 : 2 * r;  // inner rows: only the two end voxels lie on the shell
                    for (int dx = -r; dx <= r; dx += step) {
                        const int xx = x + dx;
                        if (xx < 0 || xx >= w) continue;
                        const int32_t j = __ldg(grid + (int64_t(zz) * h + yy) * w + xx);
                        if (j < 0) continue;
                        const double a = double(__ldg(pos + int64_t(j) * 3)) - p0;
                        const double b = double(__ldg(pos + int64_t(j) * 3 + 1)) - p1;
                        const double c = double(__ldg(pos + int64_t(j) * 3 + 2)) - p2;
                        // k-d tree order: ((a^2 + b^2) + c^2), no contraction into fma
                        insert3(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)), best);
                    }
                }
            }
        }
        float m;
        if (best[0] == inf) {
            m = 1e-3f;  // a lone seed
        } else {
            const float d1 = float(sqrt(best[0]));
            const float d2 = best[1] == inf ? d1 : float(sqrt(best[1]));
            const float d3 = best[2] == inf ? d2 : float(sqrt(best[2]));
            m = fmaxf(__fdiv_rn(__fadd_rn(__fadd_rn(d1, d2), d3), 3.0f), 1e-6f);
        }
        out[i] = m;
    }
}

int grid_of(int64_t n) {
    int64_t b = (n + kBlock - 1) / kBlock;
    return int(b < 1 ? 1 : (b > 65535 * 8 ? 65535 * 8 : b));
}

}  // namespace

extern "C" {

int gsv_knn3_mean_distance(const int64_t* voxels, const float* positions, int64_t n, int32_t d, int32_t h, int32_t w,
                           int32_t* grid, float* mean_distance, void* stream) {
    if (n < 0 || d <= 0 || h <= 0 || w <= 0 || (n > 0 && (!voxels || !positions || !grid || !mean_distance)) ||
        n > int64_t(INT32_MAX))
        return GSV_ERR_INVALID_ARGUMENT;
    if (n == 0) return GSV_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t vol = int64_t(d) * h * w;
    GSV_CUDA_TRY(cudaMemsetAsync(grid, 0xff, size_t(vol) * sizeof(int32_t), st));  // -1: empty voxel
    k_mark<<<grid_of(n), kBlock, 0, st>>>(voxels, n, grid);
    GSV_LAUNCH_CHECK();
    k_knn3<<<grid_of(n), kBlock, 0, st>>>(voxels, positions, n, d, h, w, grid, mean_distance);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
