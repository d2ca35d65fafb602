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

constexpr int kRowsPerBlock = 8;       // blockDim = (32, 8): lanes walk a row, warps take rows
constexpr int kResidualBlocks = 1184;  // fixed: the loss sum order does not depend on the device

struct Geo {
    int32_t d, h, w;
    int64_t v;  // d*h*w
};

// a + s (|s| < n) wrapped into [0, n): one step of fftshift / ifftshift
__device__ __forceinline__ int wrap(int a, int s, int n) {
    const int t = a + s;
    return t >= n ? t - n : (t < 0 ? t + n : t);
}

// Row r of the [nc, d, h] row space: coil, and the (d, h) row shifted by
// sign * n/2 on both axes, as the element offset of that row in a volume.
__device__ __forceinline__ void row_of(const Geo& g, int r, int sign, int& c, int64_t& own, int64_t& shifted_row) {
    const int dh = g.d * g.h;
    c = r / dh;
    const int rem = r - c * dh;
    const int a = rem / g.h, b = rem - a * g.h;
    own = int64_t(rem) * g.w;
    shifted_row = (int64_t(wrap(a, sign * (g.d / 2), g.d)) * g.h + wrap(b, sign * (g.h / 2), g.h)) * g.w;
}

__global__ void __launch_bounds__(32 * kRowsPerBlock) k_expand(const float2* __restrict__ x,
                                                              const float2* __restrict__ s, int32_t nc, Geo g,
                                                              float2* __restrict__ out) {
    const int rows = nc * g.d * g.h;
    for (int r = blockIdx.x * kRowsPerBlock + threadIdx.y; r < rows; r += gridDim.x * kRowsPerBlock) {
        int c;
        int64_t own, src;
        row_of(g, r, +1, c, own, src);  // X[c, k] = (S x)[c, k + n/2]
        const float2* sc = s + int64_t(c) * g.v;
        float2* oc = out + int64_t(c) * g.v;
        for (int w = threadIdx.x; w < g.w; w += 32) {
            const int sw = wrap(w, g.w / 2, g.w);
            const float2 a = __ldg(sc + src + sw), b = __ldg(x + src + sw);
            oc[own + w] = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        }
    }
}

__global__ void __launch_bounds__(32 * kRowsPerBlock) k_residual(float2* __restrict__ kp,
                                                                const float* __restrict__ mask,
                                                                const float2* __restrict__ y, int32_t nc, Geo g,
                                                                float* __restrict__ partial) {
    const int rows = nc * g.d * g.h;
    float acc = 0.f;
    for (int r = blockIdx.x * kRowsPerBlock + threadIdx.y; r < rows; r += gridDim.x * kRowsPerBlock) {
        int c;
        int64_t own, nat;
        row_of(g, r, +1, c, own, nat);  // Kp[c, j] is fft3c's entry [c, j + n/2]
        float2* kc = kp + int64_t(c) * g.v;
        const float2* yc = y + int64_t(c) * g.v;
        for (int w = threadIdx.x; w < g.w; w += 32) {
            const int64_t k = nat + wrap(w, g.w / 2, g.w);
            const float m = __ldg(mask + k);
            const float2 z = kc[own + w], t = __ldg(yc + k);
            const float rr = fmaf(m, z.x, -t.x), ri = fmaf(m, z.y, -t.y);
            acc = fmaf(rr, rr, fmaf(ri, ri, acc));
            kc[own + w] = make_float2(2.f * m * rr, 2.f * m * ri);
        }
    }
    // fixed-order block sum
    __shared__ float red[kRowsPerBlock];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (threadIdx.x == 0) red[threadIdx.y] = acc;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        float b = 0.f;
        for (int i = 0; i < kRowsPerBlock; ++i) b += red[i];
        partial[blockIdx.x] = b;
    }
}

__global__ void k_sum_partials(const float* __restrict__ partial, int n, float* __restrict__ loss) {
    __shared__ double red[256];
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

__global__ void __launch_bounds__(32 * kRowsPerBlock) k_adjoint(const float2* __restrict__ gk,
                                                               const float2* __restrict__ s, int32_t nc, Geo g,
                                                               float2* __restrict__ out) {
    const int rows = g.d * g.h;
    for (int r = blockIdx.x * kRowsPerBlock + threadIdx.y; r < rows; r += gridDim.x * kRowsPerBlock) {
        int c0;
        int64_t own, src;
        row_of(g, r, -1, c0, own, src);  // (S x).grad[i] = X.grad[i - n/2]
        for (int w = threadIdx.x; w < g.w; w += 32) {
            const int64_t i = own + w, k = src + wrap(w, -(g.w / 2), g.w);
            float2 a = make_float2(0.f, 0.f);
            for (int c = 0; c < nc; ++c) {
                const float2 sc = __ldg(s + c * g.v + i), z = __ldg(gk + c * g.v + k);
                a.x = fmaf(sc.x, z.x, fmaf(sc.y, z.y, a.x));  // conj(s) * z
                a.y = fmaf(sc.x, z.y, fmaf(-sc.y, z.x, a.y));
            }
            out[i] = a;
        }
    }
}

__device__ __forceinline__ float cabs(float2 z) { return sqrtf(fmaf(z.x, z.x, z.y * z.y)); }
__device__ __forceinline__ float sgn(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// TV(|x|) = sum over the three axes of |m[i + e_a] - m[i]|, m = |x|
// (3DGS/3dgsVC/losses/losses.py:18-26, MagnitudeTVLoss), and its gradient in
// torch's convention: dTV/dm_i (a sum of signs) times x_i / |x_i| (0 at 0).
__global__ void __launch_bounds__(32 * kRowsPerBlock) k_tv(const float2* __restrict__ x, Geo g,
                                                          float* __restrict__ partial, float2* __restrict__ grad) {
    const int rows = g.d * g.h;
    const int64_t sd = int64_t(g.h) * g.w, sh = g.w;
    float acc = 0.f;
    for (int r = blockIdx.x * kRowsPerBlock + threadIdx.y; r < rows; r += gridDim.x * kRowsPerBlock) {
        const int a = r / g.h, b = r - a * g.h;
        for (int c = threadIdx.x; c < g.w; c += 32) {
            const int64_t i = int64_t(r) * g.w + c;
            const float2 z = __ldg(x + i);
            const float m = cabs(z);
            float dm = 0.f;
            if (a + 1 < g.d) { const float t = cabs(__ldg(x + i + sd)) - m; acc += fabsf(t); dm -= sgn(t); }
            if (b + 1 < g.h) { const float t = cabs(__ldg(x + i + sh)) - m; acc += fabsf(t); dm -= sgn(t); }
            if (c + 1 < g.w) { const float t = cabs(__ldg(x + i + 1)) - m; acc += fabsf(t); dm -= sgn(t); }
            if (a > 0) dm += sgn(m - cabs(__ldg(x + i - sd)));
            if (b > 0) dm += sgn(m - cabs(__ldg(x + i - sh)));
            if (c > 0) dm += sgn(m - cabs(__ldg(x + i - 1)));
            grad[i] = m > 0.f ? make_float2(dm * z.x / m, dm * z.y / m) : make_float2(0.f, 0.f);
        }
    }
    __shared__ float red[kRowsPerBlock];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (threadIdx.x == 0) red[threadIdx.y] = acc;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        float t = 0.f;
        for (int i = 0; i < kRowsPerBlock; ++i) t += red[i];
        partial[blockIdx.x] = t;
    }
}

bool geo_ok(int32_t nc, int32_t d, int32_t h, int32_t w) {
    return nc > 0 && d > 0 && h > 0 && w > 0 && int64_t(nc) * d * h < (int64_t(1) << 31);
}

int grid_rows(int64_t rows) {
    int64_t b = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
    return int(b < 1 ? 1 : (b > (1 << 20) ? (1 << 20) : b));
}

}  // namespace

extern "C" {

size_t gsv_sense_workspace_bytes(void) { return size_t(kResidualBlocks) * sizeof(float); }

int gsv_sense_expand(const float* volume, const float* coils, int32_t ncoils, int32_t d, int32_t h, int32_t w,
                     float* out, void* stream) {
    if (!volume || !coils || !out || !geo_ok(ncoils, d, h, w)) return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    k_expand<<<grid_rows(int64_t(ncoils) * d * h), dim3(32, kRowsPerBlock), 0, static_cast<cudaStream_t>(stream)>>>(
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
    k_residual<<<kResidualBlocks, dim3(32, kRowsPerBlock), 0, st>>>(reinterpret_cast<float2*>(kspace), mask,
                                                   reinterpret_cast<const float2*>(measured), ncoils, g, partial);
    GSV_LAUNCH_CHECK();
    k_sum_partials<<<1, 256, 0, st>>>(partial, kResidualBlocks, loss);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_sense_adjoint(const float* kgrad_image, const float* coils, int32_t ncoils, int32_t d, int32_t h,
                      int32_t w, float* volume_grad, void* stream) {
    if (!kgrad_image || !coils || !volume_grad || !geo_ok(ncoils, d, h, w)) return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    k_adjoint<<<grid_rows(int64_t(d) * h), dim3(32, kRowsPerBlock), 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2*>(kgrad_image), reinterpret_cast<const float2*>(coils), ncoils, g,
        reinterpret_cast<float2*>(volume_grad));
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_tv_magnitude(const float* volume, int32_t d, int32_t h, int32_t w, float* loss, float* grad, void* ws,
                     size_t ws_bytes, void* stream) {
    if (!volume || !loss || !grad || !ws || ws_bytes < gsv_sense_workspace_bytes() || !geo_ok(1, d, h, w))
        return GSV_ERR_INVALID_ARGUMENT;
    const Geo g{d, h, w, int64_t(d) * h * w};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* partial = static_cast<float*>(ws);
    k_tv<<<kResidualBlocks, dim3(32, kRowsPerBlock), 0, st>>>(reinterpret_cast<const float2*>(volume), g, partial,
                                                             reinterpret_cast<float2*>(grad));
    GSV_LAUNCH_CHECK();
    k_sum_partials<<<1, 256, 0, st>>>(partial, kResidualBlocks, loss);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
