// gsv_common.cuh -- shared device code of the sm_100a tile voxelizer.
//
// The quadratic-form coefficients and the inclusion predicate are written
// with explicit round-to-nearest intrinsics (__fmul_rn / __fadd_rn /
// __fmaf_rn ...), so nvcc cannot contract or reorder them: the CPU oracle
// evaluates the very same FP32 sequence and therefore includes exactly the
// same (voxel, Gaussian) pairs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gsv.h"

namespace gsv {

// One Gaussian as the render kernels consume it: 48 bytes, three float4.
// Quadratic form in voxel units: m(e) = q00 e0^2 + q01x2 e0 e1 + q02x2 e0 e2
//                                     + q11 e1^2 + q12x2 e1 e2 + q22 e2^2,
// e = voxel - center, Q = cov_inv / (hs hs^T) (half shape hs).
struct __align__(16) Rec {
    float c0, c1, c2, q00;
    float q01x2, q02x2, q11, q12x2;
    float q22, rho_r, rho_i, pad;
};
static_assert(sizeof(Rec) == 48, "Rec must be 48 bytes");

// Number of per-(tile, Gaussian) gradient moments, padded to 12 floats:
// [0] sum w*gr  [1] sum w*gi  [2..4] sum a*e_k  [5..10] sum a*e_j*e_k
// (jk = 00,01,02,11,12,22), a = dL/dm = -0.5 w (rho_r gr + rho_i gi).
constexpr int kMom = 11;
constexpr int kMomStride = 12;

constexpr float kCut = 9.0f;                  // mahal <= 9 (tile_voxelize_cuda_kernel.cu:130)
constexpr float kNegHalfLog2e = -0.72134752044448170f;  // -0.5 * log2(e)

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// torch max-reduction semantics (NaN propagates), tile_voxelizer.py:286.
__device__ __forceinline__ float nanmax3(float a, float b, float c) {
    if (isnan(a) || isnan(b) || isnan(c)) return __int_as_float(0x7fc00000);
    float m = a > b ? a : b;
    return m > c ? m : c;
}

// Quadratic-form coefficients from (scale, quaternion), FP32, fixed order.
// R(q/(|q|+1e-8)) of tile_voxelizer.py:77-84; T = R diag(1/(s+1e-8));
// M = T T^T (:288-290); Q = M / (hs hs^T).
__device__ __forceinline__ void qcoef_from_params(const float* s, const float* q, const float ih[3],
                                                  float out[6]) {
    float n2 = __fmul_rn(q[0], q[0]);
    n2 = __fadd_rn(n2, __fmul_rn(q[1], q[1]));
    n2 = __fadd_rn(n2, __fmul_rn(q[2], q[2]));
    n2 = __fadd_rn(n2, __fmul_rn(q[3], q[3]));
    const float den = __fadd_rn(__fsqrt_rn(n2), 1e-8f);
    const float w = __fdiv_rn(q[0], den), x = __fdiv_rn(q[1], den);
    const float y = __fdiv_rn(q[2], den), z = __fdiv_rn(q[3], den);
    const float tx = 2.0f * x, ty = 2.0f * y, tz = 2.0f * z;
    float r[9];
    r[0] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(ty, y)), __fmul_rn(tz, z));
    r[1] = __fsub_rn(__fmul_rn(tx, y), __fmul_rn(tz, w));
    r[2] = __fadd_rn(__fmul_rn(tx, z), __fmul_rn(ty, w));
    r[3] = __fadd_rn(__fmul_rn(tx, y), __fmul_rn(tz, w));
    r[4] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(tx, x)), __fmul_rn(tz, z));
    r[5] = __fsub_rn(__fmul_rn(ty, z), __fmul_rn(tx, w));
    r[6] = __fsub_rn(__fmul_rn(tx, z), __fmul_rn(ty, w));
    r[7] = __fadd_rn(__fmul_rn(ty, z), __fmul_rn(tx, w));
    r[8] = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(tx, x)), __fmul_rn(ty, y));
    float si[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) si[j] = __fdiv_rn(1.0f, __fadd_rn(s[j], 1e-8f));
    float t[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = __fmul_rn(r[i * 3 + j], si[j]);
    const int ia[6] = {0, 0, 0, 1, 1, 2};
    const int ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float* ta = &t[ia[k] * 3];
        const float* tb = &t[ib[k] * 3];
        float m = __fmul_rn(ta[0], tb[0]);
        m = __fadd_rn(m, __fmul_rn(ta[1], tb[1]));
        m = __fadd_rn(m, __fmul_rn(ta[2], tb[2]));
        const float qv = __fmul_rn(__fmul_rn(m, ih[ia[k]]), ih[ib[k]]);
        out[k] = (ia[k] == ib[k]) ? qv : 2.0f * qv;
    }
}

// Same coefficients from an explicit cov_inv (reference extension input);
// symmetric part (M_ab + M_ba) * 0.5, exact for symmetric input.
__device__ __forceinline__ void qcoef_from_covinv(const float* m9, const float ih[3], float out[6]) {
    const int ia[6] = {0, 0, 0, 1, 1, 2};
    const int ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float m = __fmul_rn(__fadd_rn(m9[ia[k] * 3 + ib[k]], m9[ib[k] * 3 + ia[k]]), 0.5f);
        const float qv = __fmul_rn(__fmul_rn(m, ih[ia[k]]), ih[ib[k]]);
        out[k] = (ia[k] == ib[k]) ? qv : 2.0f * qv;
    }
}

// Conservative tight extent of the inclusion set {e : m_fp32(e) <= 9}.
//
// For the exact quadratic form of the stored FP32 coefficients, m(e) <= 9
// implies |e_a| <= 3 sqrt(S_aa) with S = Q^-1 (Schur complement bound).  The
// FP32 row evaluation used by the kernels differs from the exact form by at
// most ~6 u sum_ab |Q_ab e_a e_b| <= ~3e-5 K (u = 2^-24), where
// K = max_a Q_aa S_aa >= 1 measures anisotropy, so m_fp32 <= 9 implies
// m <= 9 (1 + 3.3e-6 K).  The extent is widened by a factor
// sqrt(1 + 1e-4 K) (30x that bound) plus 0.01 voxel for the FP32 rounding
// of c -/+ extent at the culling site.  Q not positive definite, NaN, or
// K > 1e4: infinite extent (nothing is culled).  Computed in FP64 from the
// stored coefficients, rounded up.
__device__ __forceinline__ float4 tight_extent(const float qc[6]) {
    const double q00 = qc[0], q01 = 0.5 * double(qc[1]), q02 = 0.5 * double(qc[2]);
    const double q11 = qc[3], q12 = 0.5 * double(qc[4]), q22 = qc[5];
    const double c00 = q11 * q22 - q12 * q12, c11 = q00 * q22 - q02 * q02, c22 = q00 * q11 - q01 * q01;
    const double c01 = q02 * q12 - q01 * q22, c02 = q01 * q12 - q02 * q11;
    const double det = q00 * c00 + q01 * c01 + q02 * c02;
    const float inf = __int_as_float(0x7f800000);
    if (!(q00 > 0.0 && c22 > 0.0 && det > 0.0 && c00 > 0.0 && c11 > 0.0)) return make_float4(inf, inf, inf, 0.f);
    const double s0 = c00 / det, s1 = c11 / det, s2 = c22 / det;
    double k = q00 * s0;
    k = fmax(k, q11 * s1);
    k = fmax(k, q22 * s2);
    if (!(k <= 1e4)) return make_float4(inf, inf, inf, 0.f);
    const double f = 9.0 * (1.0 + 1e-4 * k);
    return make_float4(__double2float_ru(sqrt(f * s0) + 0.01), __double2float_ru(sqrt(f * s1) + 0.01),
                       __double2float_ru(sqrt(f * s2) + 0.01), 0.f);
}

// Row terms of the quadratic form for fixed (e0, e1):
//   m(e2) = fma(fma(q22, e2, B), e2, A)
__device__ __forceinline__ float row_a(const Rec& g, float e0, float e1) {
    const float u = __fmaf_rn(g.q01x2, e1, __fmul_rn(g.q00, e0));
    return __fmaf_rn(u, e0, __fmul_rn(__fmul_rn(g.q11, e1), e1));
}
__device__ __forceinline__ float row_b(const Rec& g, float e0, float e1) {
    return __fmaf_rn(g.q12x2, e1, __fmul_rn(g.q02x2, e0));
}
__device__ __forceinline__ float row_m(float q22, float a, float b, float e2) {
    return __fmaf_rn(__fmaf_rn(q22, e2, b), e2, a);
}

// ---------------------------------------------------------------------------
// Workspace layout.  Both blobs are carved at 256-byte boundaries.
// ---------------------------------------------------------------------------

__host__ __device__ inline size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

struct GaussLayout {
    size_t rec, ext, box, counts, offsets, scan_tmp, ranges, accum, status, cs_mat, cs_pos, total;
    size_t scan_tmp_bytes;
    bool cs;  // the counting-sort binning applies (cs_mat: per-row tile counts, cs_pos: positions)
};

struct PairLayout {
    size_t keys_in, vals_in, keys_out, vals_out, sort_tmp, partials, total;
    size_t sort_tmp_bytes;
};

// Status word (first 64 bytes of the status region).
struct Status {
    int32_t flags;
    int32_t pad[15];
};

}  // namespace gsv

// Error plumbing for the C entry points.
#define GSV_CUDA_TRY(expr)                                  \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) {                            \
            gsv_detail_set_error(_e, #expr, __FILE__, __LINE__); \
            return GSV_ERR_CUDA;                            \
        }                                                   \
    } while (0)

#define GSV_LAUNCH_CHECK() GSV_CUDA_TRY(cudaGetLastError())

void gsv_detail_set_error(cudaError_t e, const char* what, const char* file, int line);
