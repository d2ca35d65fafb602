// sense_ops.cu -- fused elementwise kernels of the SENSE data-consistency
// term around the 3-D FFTs (which stay torch.fft / cuFFT).
//
// The plain 3DGSMR loss (3DGS/3dgsVC/trainers/trainer.py:256-268) is
//   L = sum_c || M * fft3c(S_c x) - y_c ||^2,
//   fft3c = fftshift o fftn(ortho) o ifftshift over the last three axes.
// Evaluated op by op it streams the [C, V] coil images through memory about
// ten times per iteration (coil product, two shifts, mask, residual, square,
// sum, and as many again in the backward).  Here the shifts are folded into
// the index arithmetic of three kernels:
//   expand  : X[c, k]  = S[c, i] x[i],            i = k + n/2 (mod n) per axis
//   residual: R[c, j]  = M[k] Kp[c, j] - y[c, k],  k = j + n/2 (mod n),
//             L = sum |R|^2 (fixed-order two-stage sum), Kp <- 2 M R in place
//             (the gradient of L with respect to Kp = fftn(X))
//   adjoint : g[i]     = sum_c conj(S[c, i]) G[c, k], k = i - n/2 (mod n),
//             G = ifftn(2 M R) (the adjoint of an orthonormal fftn)
// so that the data term costs expand + fftn + residual + ifftn + adjoint.
// g is the gradient of L with respect to x in torch's convention for
// complex tensors (conj-Wirtinger times 2: d|z|^2 -> 2 z).
#include <cuComplex.h>

#include "gsv_common.cuh"

namespace {

constexpr int kBlock = 256;
constexpr int kResidualBlocks = 1184;  // fixed: the loss sum order does not depend on the device

struct Geo {
    int32_t d, h, w;
    int64_t v;  // d*h*w
};

__device__ __forceinline__ int64_t shifted(const Geo& g, int64_t flat, int sign) {
    // (a + sign * n/2) mod n on each axis of the row-major (d, h, w) index
    const int64_t hw = int64_t(g.h) * g.w;
    int a = int(flat / hw), b = int((flat / g.w) % g.h), c = int(flat % g.w);
    a = (a + sign * (g.d / 2) + g.d) % g.d;
    b = (b + sign * (g.h / 2) + g.h) % g.h;
    c = (c + sign * (g.w / 2) + g.w) % g.w;
    return (int64_t(a) * g.h + b) * g.w + c;
}

__global__ void __launch_bounds__(kBlock) k_expand(const float2* __restrict__ x, const float2* __restrict__ s,
                                                  int32_t nc, Geo g, float2* __restrict__ out) {
    const int64_t total = int64_t(nc) * g.v;
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = e / g.v, k = e - c * g.v;
        const int64_t i = shifted(g, k, +1);
        const float2 a = __ldg(s + c * g.v + i), b = __ldg(x + i);
        out[e] = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
}

__global__ void __launch_bounds__(kBlock) k_residual(float2* __restrict__ kp, const float* __restrict__ mask,
                                                    const float2* __restrict__ y, int32_t nc, Geo g,
                                                    float* __restrict__ partial) {
    const int64_t total = int64_t(nc) * g.v;
    float acc = 0.f;
    for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = e / g.v, j = e - c * g.v;
        const int64_t k = shifted(g, j, +1);
        const float m = __ldg(mask + k);
        const float2 z = kp[e], t = __ldg(y + c * g.v + k);
        const float rr = fmaf(m, z.x, -t.x), ri = fmaf(m, z.y, -t.y);
        acc = fmaf(rr, rr, fmaf(ri, ri, acc));
        kp[e] = make_float2(2.f * m * rr, 2.f * m * ri);
    }
    // fixed-order block sum
    __shared__ float red[kBlock / 32];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.f;
        for (int i = 0; i < kBlock / 32; ++i) b += red[i];
        partial[blockIdx.x] = b;
    }
}

__global__ void k_sum_partials(const float* __restrict__ partial, int n, float* __restrict__ loss) {
    __shared__ double red[kBlock];
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += partial[i];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = float(red[0]);
}

__global__ void __launch_bounds__(kBlock) k_adjoint(const float2* __restrict__ gk, const float2* __restrict__ s,
                                                   int32_t nc, Geo g, float2* __restrict__ out) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < g.v; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t k = shifted(g, i, -1);
        float2 a = make_float2(0.f, 0.f);
        for (int c = 0; c < nc; ++c) {
            const float2 sc = __ldg(s + c * g.v + i), z = __ldg(gk + c * g.v + k);
            a.x = fmaf(sc.x, z.x, fmaf(sc.y, z.y, a.x));  // conj(s) * z
            a.y = fmaf(sc.x, z.y, fmaf(-sc.y, z.x, a.y));
        }
        out[i] = a;
    }
}

bool geo_ok(int32_t nc, int32_t d, int32_t h, int32_t w) { return nc > 0 && d > 0 && h > 0 && w > 0; }

int grid_of(int64_t n) {
    int64_t b = (n + kBlock - 1) / kBlock;
    return int(b < 1 ? 1 : (b > 65535 * 16 ? 65535 * 16 : b));
}

}  // namespace

extern "C" {

size_t gsv_sense_workspace_bytes(void) { return size_t(kResidualBlocks) * sizeof(float); }

int gsv_sense_expand(const float* volume, const float* coils, int32_t ncoils, int32_t d, int32_t h, int32_t w,
                     float* out, void* stream) {
    if (!volume || !coils || !out || !geo_ok(ncoils, d, h, w)) return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    k_expand<<<grid_of(int64_t(ncoils) * g.v), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2*>(volume), reinterpret_cast<const float2*>(coils), ncoils, g,
        reinterpret_cast<float2*>(out));
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_sense_residual(float* kspace, const float* mask, const float* measured, int32_t ncoils, int32_t d,
                       int32_t h, int32_t w, float* loss, void* ws, size_t ws_bytes, void* stream) {
    if (!kspace || !mask || !measured || !loss || !ws || ws_bytes < gsv_sense_workspace_bytes() ||
        !geo_ok(ncoils, d, h, w))
        return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* partial = static_cast<float*>(ws);
    k_residual<<<kResidualBlocks, kBlock, 0, st>>>(reinterpret_cast<float2*>(kspace), mask,
                                                   reinterpret_cast<const float2*>(measured), ncoils, g, partial);
    GSV_LAUNCH_CHECK();
    k_sum_partials<<<1, kBlock, 0, st>>>(partial, kResidualBlocks, loss);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_sense_adjoint(const float* kgrad_image, const float* coils, int32_t ncoils, int32_t d, int32_t h,
                      int32_t w, float* volume_grad, void* stream) {
    if (!kgrad_image || !coils || !volume_grad || !geo_ok(ncoils, d, h, w)) return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    k_adjoint<<<grid_of(g.v), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2*>(kgrad_image), reinterpret_cast<const float2*>(coils), ncoils, g,
        reinterpret_cast<float2*>(volume_grad));
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
