// mlp_tcgen05.cu -- BF16 tensor-core GEMM with fused epilogues for the
// warm-start MLP (sm_100a, tcgen05 + TMEM).
//
//   C[m, n] = sum_k A[m, k] * B[n, k]      (BF16 operands, FP32 accumulate)
//
// A and B are read from global memory through arbitrary (row, k) strides, so
// the same kernel serves the forward (X W^T), the input-gradient (dY W) and
// the weight-gradient (dZ^T X, split-K) products of training.  One CTA (8
// warps) owns a 128 x N tile (N = 256 or 16); K advances in chunks of 64
// through a 2-stage shared-memory ring (two CTAs per SM).  Operands whose K axis is contiguous
// are copied with 16-byte cp.async into the canonical no-swizzle K-major
// layout, operands whose row axis is contiguous (the transposed operands of
// the weight gradients) into the MN-major one (8x8 core matrices of 128 B,
// LBO = 128 B between K-adjacent and SBO = 1024 B between row-adjacent core
// matrices in both); other strides fall back to element-wise loads.  Thread
// 0 issues tcgen05.mma (M=128, N, K=16, kind::f16, BF16 x BF16 -> F32, major
// bits from the copy modes) into a TMEM accumulator once a stage has landed,
// and tcgen05.commit on the stage's mbarrier releases the buffer for the
// next copies, so loads of later stages overlap the MMAs.  The epilogue
// reads TMEM with tcgen05.ld (warp w: lanes of quarter w%4, column half
// w/4) and, for row-major outputs, transposes each 32-column chunk through
// shared memory so that stores are coalesced; the GELU' epilogue can also
// accumulate the column sums of its output (the layer's bias gradient).
// Every mbarrier wait is bounded; on time-out the kernel latches an error
// flag, skips the epilogue, waits (bounded) until the tensor-core work it
// issued has retired, frees its TMEM and returns.  gsv_mlp_gemm_test_timeout
// drives that path: thread 0 leaves one K stage's MMAs and commit out, so the
// wait on that stage runs out.
// No cluster launch, no multicast, no TMA.
#include <cuda_bf16.h>

#include "gsv_common.cuh"

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kThreads = 256;  // 8 warps: all stage operands, two column groups in the epilogue
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
    int a_mode, b_mode;    // Stage: how each operand is copied to shared memory
    float* col_sum;        // EPI_GELU_GRAD: += column sums of the BF16 output (or null)
    int* error;
    long long wait_limit;  // polls per mbarrier wait (kWaitLimit unless testing the time-out)
    int skip_stage;        // test hook: K stage whose MMAs and commit thread 0 leaves out (-1: none)
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

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
    for (long long i = 0; i < limit; ++i) {
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

// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units",
// 2016): 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), with the SFU's
// tanh.approx; its outputs are rounded to BF16, far coarser than the
// approximation.
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC0 = 0.7978845608028654f;       // sqrt(2/pi)
constexpr float kGeluC1 = 0.7978845608028654f * 0.044715f;
__device__ __forceinline__ float gelu(float x) {
    const float t = tanh_approx(x * fmaf(kGeluC1, x * x, kGeluC0));
    return 0.5f * x * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float t = tanh_approx(x * fmaf(kGeluC1, x2, kGeluC0));
    const float du = fmaf(3.0f * kGeluC1, x2, kGeluC0);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * du;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16-byte global -> shared copy that bypasses registers (cp.async, L2 only);
// bytes < 16 zero-fills the rest, bytes == 0 reads nothing.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Byte offset of element (r, k) of a staged ROWS x kBK operand tile in the
// canonical no-swizzle layouts (8x8 core matrices of 128 B):
//   K-major : (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2
//   MN-major: (r/8)*SBO + (k/8)*LBO + (k%8)*16 + (r%8)*2
// with LBO = 128 B and SBO = 1024 B in both cases, so one descriptor format
// serves both and the instruction descriptor's major bits select the
// interpretation.
__device__ __forceinline__ uint32_t tile_off(int r, int k, bool mn) {
    return (r >> 3) * kSBO + (k >> 3) * kLBO + (mn ? (k & 7) * 16 + (r & 7) * 2 : (r & 7) * 16 + (k & 7) * 2);
}

// Operand access mode, fixed per GEMM call on the host.
enum Stage : int {
    ST_K_VEC = 0,   // K contiguous (s_k == 1), 16-byte aligned rows: cp.async along K
    ST_MN_VEC = 1,  // rows contiguous (s_r == 1), 16-byte aligned K steps: cp.async along rows
    ST_SCALAR = 2   // anything else: element-wise loads, K-major layout
};

// Enqueues the copies of rows [r0, r0 + ROWS) x k [k0, k0 + kBK) of one
// operand into the stage at `dst`; out-of-range elements become zero.
// The scalar mode stores synchronously.
template <int ROWS>
__device__ __forceinline__ void stage_operand(unsigned char* dst, const __nv_bfloat16* src, long long s_r,
                                              long long s_k, int mode, int r0, int nrows, int k0, int kend) {
    const uint32_t base = smem_u32(dst);
    if (mode == ST_K_VEC) {
        constexpr int chunks = ROWS * (kBK / 8);
        for (int c = threadIdx.x; c < chunks; c += kThreads) {
            const int r = c / (kBK / 8), kc = c % (kBK / 8);
            const int gr = r0 + r, gk = k0 + kc * 8;
            const int bytes = (gr < nrows && gk < kend) ? min(16, (kend - gk) * 2) : 0;
            cp_async16(base + tile_off(r, kc * 8, false), bytes ? src + gr * s_r + gk : src, bytes);
        }
    } else if (mode == ST_MN_VEC) {
        constexpr int chunks = (ROWS / 8) * kBK;
        for (int c = threadIdx.x; c < chunks; c += kThreads) {
            const int k = c / (ROWS / 8), rg = c % (ROWS / 8);  // consecutive threads: consecutive rows
            const int gr = r0 + rg * 8, gk = k0 + k;
            const int bytes = (gr < nrows && gk < kend) ? min(16, (nrows - gr) * 2) : 0;
            cp_async16(base + tile_off(rg * 8, k, true), bytes ? src + gr + gk * s_k : src, bytes);
        }
    } else {
        constexpr int elems = ROWS * kBK;
        for (int e = threadIdx.x; e < elems; e += kThreads) {
            const int k = e / ROWS, r = e % ROWS;
            const int gr = r0 + r, gk = k0 + k;
            __nv_bfloat16 v = __float2bfloat16(0.0f);
            if (gr < nrows && gk < kend) v = src[gr * s_r + gk * s_k];
            *reinterpret_cast<__nv_bfloat16*>(dst + tile_off(r, k, false)) = v;
        }
    }
}

__device__ __forceinline__ void epi_store(const GemmArgs& g, int row, int n, float x, float bias_n) {
    const long long ci = row * g.c_sm + n * g.c_sn;
    if (g.epi == EPI_F32) {
        g.out_f32[ci] = x + bias_n;
    } else if (g.epi == EPI_BIAS_GELU) {
        x += bias_n;
        g.z_f32[ci] = x;
        g.out_bf16[ci] = __float2bfloat16(gelu(x));
    } else if (g.epi == EPI_GELU_GRAD) {
        g.out_bf16[ci] = __float2bfloat16(x * gelu_grad(g.z_f32[ci]));
    } else {
        atomicAdd(g.out_f32 + ci, x);
    }
}

__device__ __forceinline__ float bias_of(const GemmArgs& g, int n) {
    return (n < g.N && g.bias && (g.epi == EPI_F32 || g.epi == EPI_BIAS_GELU)) ? g.bias[n] : 0.f;
}

// One CTA = one 128 x BN output tile (of one K split).  All 128 threads
// stage operands with cp.async into a STAGES-deep ring; thread 0 issues the
// tcgen05.mma of a stage once every thread's copies of it have landed and
// commits it to the stage's mbarrier, which frees the buffer for the copies
// of stage kt + STAGES - 1.  The epilogue moves the accumulator out of TMEM
// 32 columns at a time and, for row-major outputs, transposes it through
// shared memory so that lanes store consecutive columns (coalesced).
template <int BN, int STAGES, int EPI>
__global__ void __launch_bounds__(kThreads, (STAGES <= 2) ? 2 : 1) k_gemm_tcgen05(const GemmArgs g) {
    constexpr int kATile = kBM * kBK * 2;   // 16 KB
    constexpr int kBTile = BN * kBK * 2;    // 32 KB for BN = 256
    constexpr int kStage = kATile + kBTile;
    constexpr uint32_t kTmemCols = BN < 32 ? 32 : BN;
    static_assert(kStage * STAGES >= kThreads * 33 * 4, "epilogue scratch must fit in the stages");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[STAGES + 1];  // one per stage + the drain barrier of the error path
    __shared__ uint32_t tmem_base_holder;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM;
    const int n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    constexpr int CW = (BN < 32) ? BN : 32;   // epilogue column chunk
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
#pragma unroll
        for (int s = 0; s <= STAGES; ++s) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_holder;
    const uint32_t idesc = make_idesc(BN) | (uint32_t(g.a_mode == ST_MN_VEC) << 15) |
                           (uint32_t(g.b_mode == ST_MN_VEC) << 16);

    auto issue = [&](int kt) {
        unsigned char* st_a = smem + (kt % STAGES) * kStage;
        const int k0 = kb + kt * kBK;
        stage_operand<kBM>(st_a, g.a, g.a_sm, g.a_sk, g.a_mode, m0, g.M, k0, ke);
        stage_operand<BN>(st_a + kATile, g.b, g.b_sn, g.b_sk, g.b_mode, n0, g.N, k0, ke);
    };
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < kt_n) issue(s);
        cp_async_commit();
    }
    bool ok = true;
    for (int kt = 0; kt < kt_n; ++kt) {
        cp_async_wait<STAGES - 2>();  // this thread's copies of stage kt have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();              // ... and everyone else's
        if (threadIdx.x == 0 && kt != g.skip_stage) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_base = smem_u32(smem + (kt % STAGES) * kStage), b_base = a_base + kATile;
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j)  // one K=16 step = two K-adjacent core matrices
                mma_bf16(tmem, make_desc(a_base + j * 2 * kLBO), make_desc(b_base + j * 2 * kLBO), idesc,
                         (kt > 0 || j > 0) ? 1u : 0u);
            mma_commit(smem_u32(&bars[kt % STAGES]));
        }
        const int nk = kt + STAGES - 1;  // refill the buffer of stage kt - 1 once its MMAs are done
        if (nk < kt_n) {
            if (kt >= 1)
                ok = mbar_wait(smem_u32(&bars[(kt - 1) % STAGES]), uint32_t(((kt - 1) / STAGES) & 1), g.wait_limit);
            if (!__syncthreads_and(ok)) break;
            issue(nk);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    if (ok && kt_n > 0)
        ok = mbar_wait(smem_u32(&bars[(kt_n - 1) % STAGES]), uint32_t(((kt_n - 1) / STAGES) & 1), g.wait_limit);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);  // also: every MMA is done with the stages, which become scratch
    if (!ok && threadIdx.x == 0) {
        atomicOr(g.error, 1);
        // A wait ran out, so MMAs committed earlier may not have been waited
        // for: one more commit arrives on the drain barrier once every
        // tcgen05 operation this thread issued has completed; TMEM is freed
        // only after that (or after the bounded wait on it gives up).
        mma_commit(smem_u32(&bars[STAGES]));
        mbar_wait(smem_u32(&bars[STAGES]), 0u, kWaitLimit);
    }

    // Epilogue: warp w reads TMEM lanes 32*(w%4).. (the rows it may access)
    // for the columns of group w/4.
    constexpr int kGroups = kThreads / 128;
    constexpr int GC = (BN / kGroups >= 16) ? BN / kGroups : BN;  // columns per group
    const int q = warp & 3, grp = warp >> 2;
    if (ok && kt_n > 0 && grp * GC < BN) {
        const uint32_t lane_addr = tmem + (uint32_t(q * 32) << 16);  // TMEM lane = accumulator row
        const int row0 = m0 + q * 32;
        const int cbeg = grp * GC, cend = cbeg + GC;
        if (g.c_sn == 1) {
            float* scr = reinterpret_cast<float*>(smem) + warp * 32 * 33;
            const int col = lane % CW, rsub = lane / CW;
            const int64_t step = int64_t(32 / CW) * g.c_sm;  // rows a lane advances per j
            for (int c0 = cbeg; c0 < cend; c0 += CW) {
                float v[CW];
                if constexpr (CW == 32) tmem_ld32(lane_addr + c0, v);
                else tmem_ld16(lane_addr + c0, v);
#pragma unroll
                for (int i = 0; i < CW; ++i) scr[lane * 33 + i] = v[i];
                __syncwarp();
                const int n = n0 + c0 + col;
                const bool n_ok = n < g.N;
                const int64_t idx0 = int64_t(row0 + rsub) * g.c_sm + n;
                if constexpr (EPI == EPI_GELU_GRAD) {
                    // all loads of the chunk in flight before the first use
                    float zv[CW];
#pragma unroll
                    for (int j = 0; j < CW; ++j) {
                        const int row = row0 + j * (32 / CW) + rsub;
                        zv[j] = (n_ok && row < g.M) ? g.z_f32[idx0 + j * step] : 0.f;
                    }
                    float cs = 0.f;
#pragma unroll
                    for (int j = 0; j < CW; ++j) {
                        const int r = j * (32 / CW) + rsub;
                        if (n_ok && row0 + r < g.M) {
                            const __nv_bfloat16 o = __float2bfloat16(scr[r * 33 + col] * gelu_grad(zv[j]));
                            g.out_bf16[idx0 + j * step] = o;
                            cs += __bfloat162float(o);
                        }
                    }
                    if (g.col_sum && n_ok) atomicAdd(g.col_sum + n, cs);
                } else {
                    const float bn = bias_of(g, n);
#pragma unroll 8
                    for (int j = 0; j < CW; ++j) {
                        const int r = j * (32 / CW) + rsub;
                        if (!(n_ok && row0 + r < g.M)) continue;
                        const int64_t ci = idx0 + j * step;
                        const float x = scr[r * 33 + col];
                        if constexpr (EPI == EPI_F32) {
                            g.out_f32[ci] = x + bn;
                        } else if constexpr (EPI == EPI_BIAS_GELU) {
                            g.z_f32[ci] = x + bn;
                            g.out_bf16[ci] = __float2bfloat16(gelu(x + bn));
                        } else {
                            atomicAdd(g.out_f32 + ci, x);
                        }
                    }
                }
                __syncwarp();
            }
        } else {
            for (int c0 = cbeg; c0 < cend; c0 += 16) {
                float v[16];
                tmem_ld16(lane_addr + c0, v);
                if (row0 + lane >= g.M) continue;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int n = n0 + c0 + i;
                    if (n >= g.N) break;
                    epi_store(g, row0 + lane, n, v[i], bias_of(g, n));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Split-K weight gradients walk long K ranges: 4 stages hide the copy
// latency there; the other products (K <= 256) keep 2 stages and 2 CTAs/SM.
template <int EPI>
int launch_gemm(const GemmArgs& g, int bn, dim3 grid, cudaStream_t st) {
    constexpr int kStages = (EPI == EPI_ATOMIC_F32) ? 4 : 2;
    if (bn == 256) {
        const int smem = kStages * (kBM * kBK * 2 + 256 * kBK * 2);
        GSV_CUDA_TRY(cudaFuncSetAttribute(k_gemm_tcgen05<256, kStages, EPI>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_gemm_tcgen05<256, kStages, EPI><<<grid, kThreads, smem, st>>>(g);
    } else {
        const int smem = kStages * (kBM * kBK * 2 + 16 * kBK * 2);
        GSV_CUDA_TRY(cudaFuncSetAttribute(k_gemm_tcgen05<16, kStages, EPI>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_gemm_tcgen05<16, kStages, EPI><<<grid, kThreads, smem, st>>>(g);
    }
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

// Operand copy mode: 16-byte cp.async needs a 16-byte aligned base and a
// contiguous axis whose neighbours sit a multiple of 8 elements apart.
int stage_mode(const void* p, long long s_r, long long s_k) {
    const bool aligned = (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    if (aligned && s_k == 1 && s_r % 8 == 0) return ST_K_VEC;
    if (aligned && s_r == 1 && s_k % 8 == 0) return ST_MN_VEC;
    return ST_SCALAR;
}

int mlp_gemm(const void* a, long long a_sm, long long a_sk, const void* b, long long b_sn, long long b_sk, int M,
             int N, int K, int splits, const float* bias, float* out_f32, void* out_bf16, float* z_f32,
             long long c_sm, long long c_sn, int epi, float* col_sum, int* error, void* stream,
             long long wait_limit, int skip_stage) {
    if (!a || !b || !error || M <= 0 || N <= 0 || K <= 0 || (N % 16) != 0 || splits <= 0) return GSV_ERR_INVALID_ARGUMENT;
    if (epi < EPI_F32 || epi > EPI_ATOMIC_F32) return GSV_ERR_INVALID_ARGUMENT;
    if (splits > 1 && epi != EPI_ATOMIC_F32) return GSV_ERR_INVALID_ARGUMENT;
    if ((epi == EPI_F32 || epi == EPI_ATOMIC_F32) && !out_f32) return GSV_ERR_INVALID_ARGUMENT;
    if ((epi == EPI_BIAS_GELU || epi == EPI_GELU_GRAD) && (!out_bf16 || !z_f32)) return GSV_ERR_INVALID_ARGUMENT;
    if (col_sum && (epi != EPI_GELU_GRAD || c_sn != 1)) return GSV_ERR_INVALID_ARGUMENT;
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
    g.c_sm = c_sm; g.c_sn = c_sn; g.epi = epi; g.col_sum = col_sum; g.error = error;
    g.wait_limit = wait_limit; g.skip_stage = skip_stage;
    g.a_mode = stage_mode(a, a_sm, a_sk);
    g.b_mode = stage_mode(b, b_sn, b_sk);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int bn = (N % 256 == 0) ? 256 : 16;
    dim3 grid((M + kBM - 1) / kBM, N / bn, zs);
    int rc = GSV_OK;
    switch (epi) {
        case EPI_F32: rc = launch_gemm<EPI_F32>(g, bn, grid, st); break;
        case EPI_BIAS_GELU: rc = launch_gemm<EPI_BIAS_GELU>(g, bn, grid, st); break;
        case EPI_GELU_GRAD: rc = launch_gemm<EPI_GELU_GRAD>(g, bn, grid, st); break;
        default: rc = launch_gemm<EPI_ATOMIC_F32>(g, bn, grid, st); break;
    }
    return rc;
}

}  // namespace

extern "C" {

int gsv_mlp_gemm(const void* a, long long a_sm, long long a_sk, const void* b, long long b_sn,
                         long long b_sk, int M, int N, int K, int splits, const float* bias, float* out_f32,
                         void* out_bf16, float* z_f32, long long c_sm, long long c_sn, int epi, float* col_sum,
                         int* error, void* stream) {
    return mlp_gemm(a, a_sm, a_sk, b, b_sn, b_sk, M, N, K, splits, bias, out_f32, out_bf16, z_f32, c_sm, c_sn, epi,
                    col_sum, error, stream, kWaitLimit, -1);
}

int gsv_mlp_gemm_test_timeout(const void* a, const void* b, int M, int N, int K, float* out_f32, int skip_stage,
                              long long wait_limit, int* error, void* stream) {
    if (skip_stage < 0 || skip_stage >= (K + kBK - 1) / kBK) return GSV_ERR_INVALID_ARGUMENT;
    if (wait_limit <= 0 || wait_limit > kWaitLimit) return GSV_ERR_INVALID_ARGUMENT;
    return mlp_gemm(a, K, 1, b, K, 1, M, N, K, 1, nullptr, out_f32, nullptr, nullptr, N, 1, EPI_F32, nullptr, error,
                    stream, wait_limit, skip_stage);
}

}  // extern "C"
