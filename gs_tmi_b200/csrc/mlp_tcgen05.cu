// mlp_tcgen05.cu -- BF16 tensor-core GEMM with fused epilogues for the
// warm-start MLP (sm_100a, tcgen05 + TMEM).
//
//   C[m, n] = sum_k A[m, k] * B[n, k]      (BF16 operands, FP32 accumulate)
//
// A and B are read from global memory through arbitrary (row, k) strides, so
// the same kernel serves the forward (X W^T), the input-gradient (dY W) and
// the weight-gradient (dZ^T X, split-K) products of training.  One CTA (4
// warps) owns a 128 x N tile (N = 256 or 16); K advances in chunks of 64
// through a two-stage shared-memory ring in the canonical no-swizzle
// K-major layout (8x8 core matrices: 16 B rows, LBO = 128 B between
// K-adjacent core matrices, SBO = 1024 B between row-adjacent ones).  Thread
// 0 issues tcgen05.mma (M=128, N, K=16, kind::f16, BF16 x BF16 -> F32) into a
// TMEM accumulator and tcgen05.commit arrives on the stage's mbarrier; the
// epilogue reads TMEM with tcgen05.ld (each warp its 32 lanes = rows).
// Every mbarrier wait is bounded; on time-out the kernel latches an error
// flag, skips the epilogue, frees its TMEM and returns.
// No cluster launch, no multicast, no TMA: operands are staged by plain
// loads (gathers and transposes included).
#include <cuda_bf16.h>

#include "gsv_common.cuh"

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kThreads = 128;
constexpr uint32_t kLBO = 128;   // bytes between K-adjacent core matrices
constexpr uint32_t kSBO = 1024;  // bytes between row-adjacent core matrices (kBK/8 * 128)
constexpr long long kWaitLimit = 1ll << 26;

enum Epi : int {
    EPI_F32 = 0,        // out_f32 = acc (+ bias)
    EPI_BIAS_GELU = 1,  // z_f32 = acc + bias; out_bf16 = gelu(z)
    EPI_GELU_GRAD = 2,  // out_bf16 = acc * gelu'(z_f32)
    EPI_ATOMIC_F32 = 3  // atomicAdd(out_f32, acc)   (split-K)
};

struct GemmArgs {
    const __nv_bfloat16* a;
    const __nv_bfloat16* b;
    long long a_sm, a_sk;  // A element (m, k) at a[m*a_sm + k*a_sk]
    long long b_sn, b_sk;  // B element (n, k) at b[n*b_sn + k*b_sk]
    int M, N, K;
    int k_per_split;       // K range per blockIdx.z
    const float* bias;     // [N] or null
    float* out_f32;
    __nv_bfloat16* out_bf16;
    float* z_f32;          // EPI_BIAS_GELU writes it, EPI_GELU_GRAD reads it
    long long c_sm, c_sn;  // C element (m, n) at c[m*c_sm + n*c_sn]
    int epi;
    int* error;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor: SWIZZLE_NONE, version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFF);
    d |= uint64_t((kLBO >> 4) & 0x3FFF) << 16;
    d |= uint64_t((kSBO >> 4) & 0x3FFF) << 32;
    d |= uint64_t(1) << 46;  // descriptor version for tcgen05
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: D=F32, A=B=BF16, both K-major, M=128.
__host__ __device__ constexpr uint32_t make_idesc(int n) {
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | (uint32_t(n >> 3) << 17)      // N / 8
           | (uint32_t(kBM >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// Stage rows [r0, r0+rows) x k [k0, k0+kBK) of a strided BF16 matrix into the
// canonical layout; out-of-range elements are zero.
template <int ROWS>
__device__ __forceinline__ void stage_tile(unsigned char* dst, const __nv_bfloat16* src, long long s_r, long long s_k,
                                           int r0, int nrows, int k0, int kend) {
    if (s_k == 1) {
        // 16-byte chunks along K (8 elements) per core-matrix row
        constexpr int chunks = ROWS * (kBK / 8);
        for (int c = threadIdx.x; c < chunks; c += kThreads) {
            const int r = c / (kBK / 8), kc = c % (kBK / 8);
            const int gr = r0 + r, gk = k0 + kc * 8;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gr < nrows) {
                const __nv_bfloat16* p = src + gr * s_r + gk;
                if (gk + 8 <= kend && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
                    v = *reinterpret_cast<const uint4*>(p);
                } else {
                    __nv_bfloat16 t[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) t[i] = (gk + i < kend) ? p[i] : __float2bfloat16(0.0f);
                    v = *reinterpret_cast<uint4*>(t);
                }
            }
            *reinterpret_cast<uint4*>(dst + (r >> 3) * kSBO + kc * kLBO + (r & 7) * 16) = v;
        }
    } else {
        // general strides (transposed operands): one element per thread step,
        // consecutive threads walk the row index (unit stride in memory)
        constexpr int elems = ROWS * kBK;
        for (int e = threadIdx.x; e < elems; e += kThreads) {
            const int k = e / ROWS, r = e % ROWS;
            const int gr = r0 + r, gk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gr < nrows && gk < kend) v = src[gr * s_r + gk * s_k];
            *reinterpret_cast<__nv_bfloat16*>(dst + (r >> 3) * kSBO + (k >> 3) * kLBO + (r & 7) * 16 + (k & 7) * 2) = v;
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_tcgen05(const GemmArgs g) {
    constexpr int kATile = kBM * kBK * 2;   // 16 KB
    constexpr int kBTile = BN * kBK * 2;    // 32 KB for BN = 256
    constexpr int kStage = kATile + kBTile;
    constexpr uint32_t kTmemCols = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base_holder;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM;
    const int n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    const int ke = min(g.K, kb + g.k_per_split);
    const int kt_n = (ke - kb + kBK - 1) / kBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_holder;
    constexpr uint32_t idesc = make_idesc(BN);
    bool ok = true;

    for (int kt = 0; kt < kt_n; ++kt) {
        const int s = kt & 1;
        if (kt >= 2) ok = ok && mbar_wait(smem_u32(&bars[s]), uint32_t(((kt - 2) >> 1) & 1));
        unsigned char* st_a = smem + s * kStage;
        unsigned char* st_b = st_a + kATile;
        const int k0 = kb + kt * kBK;
        stage_tile<kBM>(st_a, g.a, g.a_sm, g.a_sk, m0, g.M, k0, ke);
        stage_tile<BN>(st_b, g.b, g.b_sn, g.b_sk, n0, g.N, k0, ke);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_base = smem_u32(st_a), b_base = smem_u32(st_b);
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j) {
                // one K=16 step = two K-adjacent core matrices
                mma_bf16(tmem, make_desc(a_base + j * 2 * kLBO), make_desc(b_base + j * 2 * kLBO), idesc,
                         (kt > 0 || j > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&bars[s]));
        }
    }
    if (kt_n > 0) ok = ok && mbar_wait(smem_u32(&bars[(kt_n - 1) & 1]), uint32_t(((kt_n - 1) >> 1) & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok && lane == 0) atomicOr(g.error, 1);

    if (ok && kt_n > 0) {
        const int row = m0 + warp * 32 + lane;  // TMEM lane = accumulator row
        const uint32_t lane_addr = tmem + (uint32_t(warp * 32) << 16);
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(lane_addr + c0, v);
            if (row >= g.M) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int n = n0 + c0 + i;
                if (n >= g.N) break;
                const long long ci = row * g.c_sm + n * g.c_sn;
                float x = v[i];
                if (g.epi == EPI_F32) {
                    if (g.bias) x += g.bias[n];
                    g.out_f32[ci] = x;
                } else if (g.epi == EPI_BIAS_GELU) {
                    if (g.bias) x += g.bias[n];
                    g.z_f32[ci] = x;
                    g.out_bf16[ci] = __float2bfloat16(gelu(x));
                } else if (g.epi == EPI_GELU_GRAD) {
                    g.out_bf16[ci] = __float2bfloat16(x * gelu_grad(g.z_f32[ci]));
                } else {
                    atomicAdd(g.out_f32 + ci, x);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace

extern "C" {

int gsv_mlp_gemm(const void* a, long long a_sm, long long a_sk, const void* b, long long b_sn,
                         long long b_sk, int M, int N, int K, int splits, const float* bias, float* out_f32,
                         void* out_bf16, float* z_f32, long long c_sm, long long c_sn, int epi, int* error,
                         void* stream) {
    if (!a || !b || !error || M <= 0 || N <= 0 || K <= 0 || (N % 16) != 0 || splits <= 0) return GSV_ERR_INVALID_ARGUMENT;
    if (epi < EPI_F32 || epi > EPI_ATOMIC_F32) return GSV_ERR_INVALID_ARGUMENT;
    if (splits > 1 && epi != EPI_ATOMIC_F32) return GSV_ERR_INVALID_ARGUMENT;
    if ((epi == EPI_F32 || epi == EPI_ATOMIC_F32) && !out_f32) return GSV_ERR_INVALID_ARGUMENT;
    if ((epi == EPI_BIAS_GELU || epi == EPI_GELU_GRAD) && (!out_bf16 || !z_f32)) return GSV_ERR_INVALID_ARGUMENT;
    GemmArgs g{};
    g.a = static_cast<const __nv_bfloat16*>(a);
    g.b = static_cast<const __nv_bfloat16*>(b);
    g.a_sm = a_sm; g.a_sk = a_sk; g.b_sn = b_sn; g.b_sk = b_sk;
    g.M = M; g.N = N; g.K = K;
    const int kchunks = (K + kBK - 1) / kBK;
    const int per = (kchunks + splits - 1) / splits;
    g.k_per_split = per * kBK;
    const int zs = (K + g.k_per_split - 1) / g.k_per_split;
    g.bias = bias; g.out_f32 = out_f32; g.out_bf16 = static_cast<__nv_bfloat16*>(out_bf16); g.z_f32 = z_f32;
    g.c_sm = c_sm; g.c_sn = c_sn; g.epi = epi; g.error = error;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int bn = (N % 256 == 0) ? 256 : 16;
    dim3 grid((M + kBM - 1) / kBM, N / bn, zs);
    if (bn == 256) {
        const int smem = 2 * (kBM * kBK * 2 + 256 * kBK * 2);
        GSV_CUDA_TRY(cudaFuncSetAttribute(k_gemm_tcgen05<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_gemm_tcgen05<256><<<grid, kThreads, smem, st>>>(g);
    } else {
        const int smem = 2 * (kBM * kBK * 2 + 16 * kBK * 2);
        GSV_CUDA_TRY(cudaFuncSetAttribute(k_gemm_tcgen05<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_gemm_tcgen05<16><<<grid, kThreads, smem, st>>>(g);
    }
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
