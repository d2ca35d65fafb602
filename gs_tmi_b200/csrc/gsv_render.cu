// gsv_render.cu -- forward / backward tile kernels and the gradient finalize.
//
// Work decomposition (tile edge 8, the reference default):
//   one CTA of 4 warps per tile; every warp covers the whole 8x8x8 tile
//   (lane l owns the two 8-voxel rows (d0+l/8, h0+l%8) and (d0+4+l/8, h0+l%8))
//   and the tile's Gaussian list is dealt out to the warps position by
//   position (warp w takes positions w, w+4, ...).  A warp stages up to 32
//   of its Gaussians in shared memory, drops those whose tight extent
//   misses the CTA's voxels, then walks the rest; for
//   each Gaussian a lane evaluates its 16 voxels with the row form
//   m = fma(fma(q22, e2, B), e2, A) (A, B once per row), and the exp / FMA
//   part runs only when some lane of the warp is inside the 3-sigma cutoff.
//   Forward: per-warp partial tiles are summed through shared memory once
//   per tile and stored as complex64.  Backward: per (tile, Gaussian) a
//   lane folds its voxels into 11 moments, the warp reduce-scatters them
//   (16 shuffles) and lanes issue one atomic per moment (or, deterministic,
//   write the per-pair partial for a fixed-order reduction in finalize).
//
// Other tile edges use a generic one-voxel-per-thread kernel pair.
//
// Reference semantics (3DGS/3dgsVC/gaussian/cuda_ext/tile_voxelize_cuda_kernel.cu):
//   forward  :118-141  vol = sum_{g in list(tile), m <= 9} exp(-m/2) rho_g
//   backward :217-252  dL/drho, dL/dcenter, dL/dcov_inv for included pairs
#include <cstdio>

#include "gsv_common.cuh"

using namespace gsv;

namespace gsv {
int layout_for(gsv_shape shape, int64_t n, int64_t cap, int flags, GaussLayout* G, PairLayout* P,
               int64_t* ntiles);
}

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;
constexpr int kThreads = kWarps * 32;

struct RenderArgs {
    // native Gaussians
    const Rec* recs;
    const float4* ext;  // conservative tight extent of each inclusion set (voxels)
    // reference-compatible Gaussians
    const float* centers;
    const float* cov_inv;
    const float* den_r;
    const float* den_i;
    const float* half_shape;
    // binning
    const int2* ranges;
    const int32_t* pair_ids;
    int32_t d, h, w, ts, nth, ntw;
    int64_t ntiles;
    float hs[3], ih[3];  // native half shape and its reciprocal
    // forward outputs
    float* vol;    // complex64 interleaved
    float* vol_r;  // planar
    float* vol_i;
    // backward inputs / outputs
    const float* gvol;  // complex64 interleaved
    const float* gv_r;  // planar
    const float* gv_i;
    float* accum;     // [n, 12] moments (native, atomics)
    float* partials;  // [pairs, 12] moments (native, deterministic), at each pair's emission index
    const int64_t* offsets;  // per-Gaussian first emission index (binning scan)
    int64_t capacity;        // pair capacity (bound of every emission index)
    float* g_center;  // compat outputs
    float* g_cov;
    float* g_dr;
    float* g_di;
    int chunk;  // Gaussians staged per warp chunk (<= 32)
    int cull;   // skip Gaussians / row slots outside the tight extent
    int split;  // backward: CTAs sharing one (half) tile's list, each taking every split-th quarter
    // finalize
    gsv_params prm;
    gsv_grads grd;
    const int4* boxes;
};

template <bool COMPAT>
__device__ __forceinline__ void compat_ih(const RenderArgs& a, float ih[3]) {
    if (COMPAT) {
#pragma unroll
        for (int k = 0; k < 3; ++k) ih[k] = __fdiv_rn(1.0f, __ldg(a.half_shape + k));
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) ih[k] = a.ih[k];
    }
}

template <bool COMPAT>
__device__ __forceinline__ Rec load_rec(const RenderArgs& a, int gid, const float ih[3]) {
    Rec r;
    if (!COMPAT) {
        const float4* p = reinterpret_cast<const float4*>(a.recs + gid);
        const float4 x = __ldg(p), y = __ldg(p + 1), z = __ldg(p + 2);
        r.c0 = x.x; r.c1 = x.y; r.c2 = x.z; r.q00 = x.w;
        r.q01x2 = y.x; r.q02x2 = y.y; r.q11 = y.z; r.q12x2 = y.w;
        r.q22 = z.x; r.rho_r = z.y; r.rho_i = z.z; r.pad = 0.0f;
    } else {
        float m9[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) m9[k] = __ldg(a.cov_inv + int64_t(gid) * 9 + k);
        float qc[6];
        qcoef_from_covinv(m9, ih, qc);
        r.c0 = __ldg(a.centers + int64_t(gid) * 3);
        r.c1 = __ldg(a.centers + int64_t(gid) * 3 + 1);
        r.c2 = __ldg(a.centers + int64_t(gid) * 3 + 2);
        r.q00 = qc[0]; r.q01x2 = qc[1]; r.q02x2 = qc[2]; r.q11 = qc[3]; r.q12x2 = qc[4]; r.q22 = qc[5];
        r.rho_r = __ldg(a.den_r + gid);
        r.rho_i = __ldg(a.den_i + gid);
        r.pad = 0.0f;
    }
    return r;
}

__device__ __forceinline__ void decode_tile(const RenderArgs& a, int64_t tile, int& d0, int& h0, int& w0) {
    const int64_t per = int64_t(a.nth) * a.ntw;
    d0 = int(tile / per) * a.ts;
    const int64_t rem = tile % per;
    h0 = int(rem / a.ntw) * a.ts;
    w0 = int(rem % a.ntw) * a.ts;
}

// Reduce-scatter of 16 per-lane values over the warp: afterwards lane l
// holds the warp total of value (l >> 1) in v[0] (lanes l and l^1 agree).
__device__ __forceinline__ float warp_reduce_scatter16(float v[16], int lane) {
    {
        const bool hi = lane & 16;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float send = hi ? v[i] : v[i + 8];
            const float keep = hi ? v[i + 8] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 16);
        }
    }
    {
        const bool hi = lane & 8;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float send = hi ? v[i] : v[i + 4];
            const float keep = hi ? v[i + 4] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 8);
        }
    }
    {
        const bool hi = lane & 4;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const float send = hi ? v[i] : v[i + 2];
            const float keep = hi ? v[i + 2] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 4);
        }
    }
    {
        const bool hi = lane & 2;
        const float send = hi ? v[0] : v[1];
        const float keep = hi ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(kFull, send, 2);
    }
    return v[0] + __shfl_xor_sync(kFull, v[0], 1);
}

// Reduce-scatter of the 11 moments (v[11] must be 0) over the warp in 13
// shuffles: afterwards lanes l and l^1 hold the warp total of moment
// moment12(l) = 6*b4 + 3*b3 + 2*b2 + b1 (b_k = bit k of l), where a value of
// 3 for 2*b2 + b1 is padding (the moment then reads as -1).
__device__ __forceinline__ float warp_reduce_scatter12(float v[12], int lane) {
    {
        const bool hi = lane & 16;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const float send = hi ? v[i] : v[i + 6];
            const float keep = hi ? v[i + 6] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 16);
        }
    }
    {
        const bool hi = lane & 8;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float send = hi ? v[i] : v[i + 3];
            const float keep = hi ? v[i + 3] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 8);
        }
    }
    {
        const bool hi = lane & 4;  // group of 3 -> pairs {0, 1} and {2, pad}
        const float send0 = hi ? v[0] : v[2], keep0 = hi ? v[2] : v[0];
        const float send1 = hi ? v[1] : 0.f, keep1 = hi ? 0.f : v[1];
        v[0] = keep0 + __shfl_xor_sync(kFull, send0, 4);
        v[1] = keep1 + __shfl_xor_sync(kFull, send1, 4);
    }
    {
        const bool hi = lane & 2;
        const float send = hi ? v[0] : v[1];
        const float keep = hi ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(kFull, send, 2);
    }
    return v[0] + __shfl_xor_sync(kFull, v[0], 1);
}

__device__ __forceinline__ int moment12(int lane) {
    const int sub = ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    return sub == 3 ? -1 : ((lane >> 4) & 1) * 6 + ((lane >> 3) & 1) * 3 + sub;
}

// Compat outputs for one (tile, Gaussian): every lane holds `tot` (lane 2i
// holds moment i); lanes 0..13 issue one atomic each.
__device__ __forceinline__ void compat_emit(const RenderArgs& a, const Rec& g, int gid, float tot,
                                            int lane, const float ih[3]) {
    float m[kMom];
#pragma unroll
    for (int i = 0; i < kMom; ++i) m[i] = __shfl_sync(kFull, tot, 2 * i);
    float out;
    switch (lane) {
        case 0: out = m[0]; break;
        case 1: out = m[1]; break;
        // dL/dcenter_a = -2 sum_b Q_ab S1_b   (reference: -2 (M d)_a / hs_a, .cu:241-243)
        case 2: out = -(2.0f * g.q00 * m[2] + g.q01x2 * m[3] + g.q02x2 * m[4]); break;
        case 3: out = -(g.q01x2 * m[2] + 2.0f * g.q11 * m[3] + g.q12x2 * m[4]); break;
        case 4: out = -(g.q02x2 * m[2] + g.q12x2 * m[3] + 2.0f * g.q22 * m[4]); break;
        // dL/dcov_inv_ab = sum a d_a d_b = S2_ab / (hs_a hs_b)  (.cu:244-252)
        case 5: out = m[5] * ih[0] * ih[0]; break;
        case 6: case 8: out = m[6] * ih[0] * ih[1]; break;
        case 7: case 11: out = m[7] * ih[0] * ih[2]; break;
        case 9: out = m[8] * ih[1] * ih[1]; break;
        case 10: case 12: out = m[9] * ih[1] * ih[2]; break;
        case 13: out = m[10] * ih[2] * ih[2]; break;
        default: out = 0.0f; break;
    }
    if (lane == 0) atomicAdd(a.g_dr + gid, out);
    else if (lane == 1) atomicAdd(a.g_di + gid, out);
    else if (lane < 5) atomicAdd(a.g_center + int64_t(gid) * 3 + (lane - 2), out);
    else if (lane < 14) {
        // lanes 5..13 -> cov entries 0..8 in row-major order
        const int e = lane - 5;
        atomicAdd(a.g_cov + int64_t(gid) * 9 + e, out);
    }
}

// ---------------------------------------------------------------------------
// Tile edge 8: forward
// ---------------------------------------------------------------------------

struct __align__(16) WarpStage {
    Rec rec[32];
    float4 e2[32][2];
    int32_t gid[32];
    int32_t meta[32];  // bit r: row slot r may hold included voxels; bits 8+: index in the chunk
    int32_t pidx[32];  // deterministic backward: emission index of the (tile, Gaussian) pair
};

// Emission index of the pair (Gaussian gid, tile (td, th, tw)): the
// Gaussian's first index plus the tile's raster position in its tile box --
// where binning emitted it.  Per-pair partials stored at this index lie
// contiguously per Gaussian, in tile raster order.
__device__ __forceinline__ int64_t emission_index(const RenderArgs& a, int gid, int td, int th, int tw) {
    const int4 b = __ldg(a.boxes + gid);
    const int t0 = b.x & 0xffff, t1 = (b.x >> 16) & 0xffff, t2 = b.y & 0xffff;
    const int n1 = b.z & 0xffff, n2 = (b.z >> 16) & 0xffff;
    return __ldg(a.offsets + gid) + (int64_t(td - t0) * n1 + (th - t1)) * n2 + (tw - t2);
}

// Execution shape of a CTA on an 8^3 binning tile.  RPL (rows per lane) = 2:
// the CTA covers the whole tile, lane l owns rows (d0+l/8, h0+l%8) and
// (d0+4+l/8, h0+l%8).  RPL = 1: the CTA covers the 4x8x8 half `sub` of the
// tile, lane l owns row (d0+4*sub+l/8, h0+l%8).  Either way each warp walks
// its share of the tile's Gaussian list (every 4th position) in chunks of
// `a.chunk` (<= 32).
constexpr int kFwdSmem = kWarps * 16 * 32 * sizeof(float2);
static_assert(sizeof(WarpStage) * kWarps <= kFwdSmem, "stage too large");

// Stages list positions base, base + kWarps, ..., (cnt of them: warp w of
// a CTA walks positions w, w + 4, w + 8, ... so the warps' shares differ by
// at most one Gaussian) and returns how many were kept.  Native layout: a Gaussian is kept only if its conservative
// tight extent (see tight_extent) reaches the CTA's rows, and it carries
// one bit per row slot it reaches; a dropped Gaussian or slot has m > 9 at
// every voxel there, so skipping it changes no sum.  The kept Gaussians keep
// their list order.  The native layout reads the extent k_prepare stored,
// the compat layout (cov_inv input) computes it here.
template <bool COMPAT, int RPL, bool DET = false>
__device__ __forceinline__ int stage_chunk(const RenderArgs& a, WarpStage& S, int base, int stride, int cnt, int lane,
                                           int d0, int h0, int w0, int sub, const float ih[3]) {
    Rec r;
    int gid = 0, bits = 0;
    if (lane < cnt) {
        gid = __ldg(a.pair_ids + base + stride * lane);
        r = load_rec<COMPAT>(a, gid, ih);
        if (!a.cull) {
            bits = (1 << RPL) - 1;
        } else {
            // native layout: precomputed by k_prepare; compat: from the
            // coefficients just derived from cov_inv (same rule)
            float4 x;
            if (COMPAT) {
                const float qc[6] = {r.q00, r.q01x2, r.q02x2, r.q11, r.q12x2, r.q22};
                x = tight_extent(qc);
            } else {
                x = __ldg(a.ext + gid);
            }
            const bool hw = __fsub_rn(r.c1, x.y) <= float(h0 + 7) && __fadd_rn(r.c1, x.y) >= float(h0) &&
                            __fsub_rn(r.c2, x.z) <= float(w0 + 7) && __fadd_rn(r.c2, x.z) >= float(w0);
            const float lo = __fsub_rn(r.c0, x.x), hi = __fadd_rn(r.c0, x.x);
#pragma unroll
            for (int k = 0; k < RPL; ++k) {
                const int ds = d0 + 4 * (k + sub);
                if (hw && lo <= float(ds + 3) && hi >= float(ds)) bits |= 1 << k;
            }
        }
    }
    const unsigned keep = __ballot_sync(kFull, bits != 0);
    if (DET && lane < cnt && !bits) {  // dropped pair: its partial is zero
        float4* dst = reinterpret_cast<float4*>(a.partials +
                                                emission_index(a, gid, d0 >> 3, h0 >> 3, w0 >> 3) * kMomStride);
        dst[0] = dst[1] = dst[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (bits) {
        const int pos = __popc(keep & ((1u << lane) - 1u));
        S.rec[pos] = r;
        S.gid[pos] = gid;
        S.meta[pos] = bits | (lane << 8);
        if (DET) S.pidx[pos] = int32_t(emission_index(a, gid, d0 >> 3, h0 >> 3, w0 >> 3));
        float e2[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) e2[k] = __fsub_rn(float(w0 + k), r.c2);
        S.e2[pos][0] = make_float4(e2[0], e2[1], e2[2], e2[3]);
        S.e2[pos][1] = make_float4(e2[4], e2[5], e2[6], e2[7]);
    }
    return __popc(keep);
}

// Forward of one tile (RPL = 2) or half tile (RPL = 1).  Two CTA barriers:
// every thread of the CTA must call it for the same (tile, sub).
template <bool COMPAT, bool PLANAR, int RPL>
__device__ __forceinline__ void forward_tile(const RenderArgs& a, int64_t tile, int sub, unsigned char* smem_raw) {
    constexpr int NV = RPL * 8;  // voxels per lane
    WarpStage* stage = reinterpret_cast<WarpStage*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    const int2 rg = a.ranges[tile];
    const int chunk = a.chunk;

    float accR[NV], accI[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) accR[k] = accI[k] = 0.0f;

    if (rg.x < rg.y) {
        float ih[3];
        compat_ih<COMPAT>(a, ih);
        float ev0[RPL];
#pragma unroll
        for (int r = 0; r < RPL; ++r) ev0[r] = float(d0 + (lane >> 3) + 4 * (r + sub));
        const float ev1 = float(h0 + (lane & 7));
        WarpStage& S = stage[warp];
        const int mine = (rg.y - rg.x - warp + kWarps - 1) / kWarps;  // list positions of this warp
        for (int i0 = 0; i0 < mine; i0 += chunk) {
            const int base = rg.x + warp + kWarps * i0;
            const int kept =
                stage_chunk<COMPAT, RPL>(a, S, base, kWarps, min(chunk, mine - i0), lane, d0, h0, w0, sub, ih);
            __syncwarp();
            for (int j = 0; j < kept; ++j) {
                const Rec g = S.rec[j];
                const int bits = S.meta[j];  // warp-uniform
                const float4 ea = S.e2[j][0], eb = S.e2[j][1];
                const float e2[8] = {ea.x, ea.y, ea.z, ea.w, eb.x, eb.y, eb.z, eb.w};
                const float e1 = __fsub_rn(ev1, g.c1);
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    if (!(bits & (1 << r))) continue;  // slot out of the Gaussian's extent
                    const float e0 = __fsub_rn(ev0[r], g.c0);
                    const float A = row_a(g, e0, e1), B = row_b(g, e0, e1);
                    float m[8];
                    bool any = false;
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        m[k] = row_m(g.q22, A, B, e2[k]);
                        any |= (m[k] <= kCut);
                    }
                    // the exp / FMA part of the slot runs only if some lane needs it
                    if (__any_sync(kFull, any)) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            if (m[k] <= kCut) {
                                const float wgt = ex2_approx(m[k] * kNegHalfLog2e);
                                accR[r * 8 + k] = fmaf(wgt, g.rho_r, accR[r * 8 + k]);
                                accI[r * 8 + k] = fmaf(wgt, g.rho_i, accI[r * 8 + k]);
                            }
                        }
                    }
                }
            }
            __syncwarp();
        }
    }

    // Sum the warps' partial (half) tiles: red[(warp*NV + k)*32 + lane].
    __syncthreads();
    float2* red = reinterpret_cast<float2*>(smem_raw);
#pragma unroll
    for (int k = 0; k < NV; ++k) red[(warp * NV + k) * 32 + lane] = make_float2(accR[k], accI[k]);
    __syncthreads();

    // Thread t stores VPT consecutive voxels of one row.
    constexpr int VPT = 2 * RPL, TPR = 8 / VPT;
    const int t = threadIdx.x;
    const int row = t / TPR;  // 0 .. 32*RPL-1
    const int lw0 = (t % TPR) * VPT;
    const int src_lane = row & 31, slot = row >> 5;
    float2 v[VPT];
#pragma unroll
    for (int i = 0; i < VPT; ++i) {
        const int k = slot * 8 + lw0 + i;
        float2 s = make_float2(0.f, 0.f);
#pragma unroll
        for (int wv = 0; wv < kWarps; ++wv) {
            const float2 x = red[(wv * NV + k) * 32 + src_lane];
            s.x += x.x;
            s.y += x.y;
        }
        v[i] = s;
    }
    const int gd = d0 + (src_lane >> 3) + 4 * (slot + sub), gh = h0 + (src_lane & 7), gw = w0 + lw0;
    if (gd >= a.d || gh >= a.h) return;
    const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + gw;
    if (PLANAR) {
#pragma unroll
        for (int i = 0; i < VPT; ++i)
            if (gw + i < a.w) {
                a.vol_r[flat + i] = v[i].x;
                a.vol_i[flat + i] = v[i].y;
            }
    } else {
        float2* out = reinterpret_cast<float2*>(a.vol) + flat;
        if (gw + VPT - 1 < a.w && (a.w & 1) == 0) {
            float4* o4 = reinterpret_cast<float4*>(out);
#pragma unroll
            for (int i = 0; i < VPT / 2; ++i)
                o4[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
        } else {
#pragma unroll
            for (int i = 0; i < VPT; ++i)
                if (gw + i < a.w) out[i] = v[i];
        }
    }
}

template <bool COMPAT, bool PLANAR, int RPL>
__global__ void __launch_bounds__(kThreads) k_forward8(const RenderArgs a) {
    __shared__ __align__(16) unsigned char smem_raw[kFwdSmem];
    constexpr int subs = 2 / RPL;
    forward_tile<COMPAT, PLANAR, RPL>(a, blockIdx.x / subs, blockIdx.x % subs, smem_raw);
}

// ---------------------------------------------------------------------------
// Tile edge 8: backward
// ---------------------------------------------------------------------------

// Backward of one tile (RPL = 2) or half tile (RPL = 1); warp-synchronous
// only.  The deterministic mode writes one partial per (tile, Gaussian) and
// therefore runs with RPL = 2 only.
template <bool COMPAT, bool DET, int RPL>
__device__ __forceinline__ void backward_tile(const RenderArgs& a, int64_t tile, int sub, WarpStage* stage,
                                              int part) {
    static_assert(!DET || RPL == 2, "deterministic partials need the whole tile in one CTA");
    constexpr int NV = RPL * 8;
    const int2 rg = a.ranges[tile];
    if (rg.x >= rg.y) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    float ih[3];
    compat_ih<COMPAT>(a, ih);
    const int chunk = a.chunk;

    // Upstream gradient of the lane's voxels (zero outside the volume).
    float gr[NV], gi[NV];
    {
        const int gh = h0 + (lane & 7);
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
            const int gd = d0 + (lane >> 3) + 4 * (r + sub);
            const bool row_ok = gd < a.d && gh < a.h;
            const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + w0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const bool ok = row_ok && (w0 + k < a.w);
                if (COMPAT) {
                    gr[r * 8 + k] = ok ? __ldg(a.gv_r + flat + k) : 0.0f;
                    gi[r * 8 + k] = ok ? __ldg(a.gv_i + flat + k) : 0.0f;
                } else {
                    const float2 x = ok ? __ldg(reinterpret_cast<const float2*>(a.gvol) + flat + k)
                                        : make_float2(0.f, 0.f);
                    gr[r * 8 + k] = x.x;
                    gi[r * 8 + k] = x.y;
                }
            }
        }
    }

    float ev0[RPL];
#pragma unroll
    for (int r = 0; r < RPL; ++r) ev0[r] = float(d0 + (lane >> 3) + 4 * (r + sub));
    const float ev1 = float(h0 + (lane & 7));
    WarpStage& S = stage[warp];
    // list positions of this warp: first, first + stride, ... (part `part` of a.split CTAs)
    const int stride = kWarps * a.split, first = part * kWarps + warp;
    const int mine = rg.y - rg.x > first ? (rg.y - rg.x - first + stride - 1) / stride : 0;
    for (int i0 = 0; i0 < mine; i0 += chunk) {
        const int base = rg.x + first + stride * i0;
        const int kept =
            stage_chunk<COMPAT, RPL, DET>(a, S, base, stride, min(chunk, mine - i0), lane, d0, h0, w0, sub, ih);
        __syncwarp();
        for (int j = 0; j < kept; ++j) {
            const Rec g = S.rec[j];
            const int bits = S.meta[j];  // warp-uniform
            const float4 ea = S.e2[j][0], eb = S.e2[j][1];
            const float e2[8] = {ea.x, ea.y, ea.z, ea.w, eb.x, eb.y, eb.z, eb.w};
            const float e1 = __fsub_rn(ev1, g.c1);
            const float hr = -0.5f * g.rho_r, hi = -0.5f * g.rho_i;
            // per row: Dr/Di = sum w g_r / g_i; R1/R2 = sum a e2 / a e2^2 with
            // a = w (hr g_r + hi g_i); sum a itself = hr Dr + hi Di (after the loop)
            float e0[RPL], Dr[RPL], Di[RPL], R1[RPL], R2[RPL];
            bool wany = false;
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                e0[r] = __fsub_rn(ev0[r], g.c0);
                Dr[r] = Di[r] = R1[r] = R2[r] = 0.f;
                if (!(bits & (1 << r))) continue;  // slot out of the Gaussian's extent
                const float A = row_a(g, e0[r], e1), B = row_b(g, e0[r], e1);
                float m[8];
                bool any = false;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    m[k] = row_m(g.q22, A, B, e2[k]);
                    any |= (m[k] <= kCut);
                }
                if (!__any_sync(kFull, any)) continue;  // warp-uniform row-slot skip
                wany = true;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int q = r * 8 + k;
                    if (m[k] <= kCut) {
                        const float wgt = ex2_approx(m[k] * kNegHalfLog2e);
                        Dr[r] = fmaf(wgt, gr[q], Dr[r]);
                        Di[r] = fmaf(wgt, gi[q], Di[r]);
                        const float ae = wgt * fmaf(hi, gi[q], hr * gr[q]) * e2[k];
                        R1[r] += ae;
                        R2[r] = fmaf(ae, e2[k], R2[r]);
                    }
                }
            }
            if (!wany) {  // no included voxel here: the pair's partial is zero
                if (DET && lane == 0) {
                    float4* dst = reinterpret_cast<float4*>(a.partials + int64_t(S.pidx[j]) * kMomStride);
                    dst[0] = dst[1] = dst[2] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                continue;
            }
            float v[16];
            float Drs = 0.f, Dis = 0.f, R0s = 0.f, R1s = 0.f, R2s = 0.f, S1 = 0.f, S2 = 0.f, S3 = 0.f;
            float R0[RPL];
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                R0[r] = fmaf(hi, Di[r], hr * Dr[r]);
                Drs += Dr[r];
                Dis += Di[r];
                R0s += R0[r];
                R1s += R1[r];
                R2s += R2[r];
                S1 = fmaf(e0[r], R0[r], S1);          // sum a e0
                S2 = fmaf(e0[r] * e0[r], R0[r], S2);  // sum a e0^2
                S3 = fmaf(e0[r], R1[r], S3);          // sum a e0 e2
            }
            v[0] = Drs;
            v[1] = Dis;
            v[2] = S1;
            v[3] = e1 * R0s;
            v[4] = R1s;
            v[5] = S2;
            v[6] = e1 * S1;
            v[7] = S3;
            v[8] = (e1 * e1) * R0s;
            v[9] = e1 * R1s;
            v[10] = R2s;
            const int gid = S.gid[j];
            if (COMPAT) {
#pragma unroll
                for (int i = 11; i < 16; ++i) v[i] = 0.f;
                compat_emit(a, g, gid, warp_reduce_scatter16(v, lane), lane, ih);
            } else {
                v[11] = 0.f;
                const float tot = warp_reduce_scatter12(v, lane);
                const int mi = moment12(lane);
                if (!(lane & 1) && mi >= 0 && mi < kMom) {
                    if (DET) a.partials[int64_t(S.pidx[j]) * kMomStride + mi] = tot;
                    else atomicAdd(a.accum + int64_t(gid) * kMomStride + mi, tot);
                }
            }
        }
        __syncwarp();
    }
}

template <bool COMPAT, bool DET, int RPL>
// Register cap: 6 resident CTAs per SM for whole tiles (80 registers), 7 for
// half tiles (72); a few spilled bytes outside the inner loop cost less
// than the occupancy they buy (measured on B200).
__global__ void __launch_bounds__(kThreads, RPL == 2 ? 6 : 7) k_backward8(const RenderArgs a) {
    __shared__ __align__(16) WarpStage stage[kWarps];
    constexpr int subs = 2 / RPL;
    const int part = blockIdx.x % a.split, rest = blockIdx.x / a.split;
    backward_tile<COMPAT, DET, RPL>(a, rest / subs, rest % subs, stage, part);
}

// ---------------------------------------------------------------------------
// Tile edge 4: one warp per 4^3 tile (four tiles per CTA, no CTA barrier).
// Lane l owns the voxel pair (d0 + l/8, h0 + (l/2)%4, w0 + 2(l%2) + {0,1});
// the warp stages up to 32 of its tile's Gaussians at a time, drops those
// whose tight extent misses the tile, and evaluates the rest with the row
// form (A, B once per lane) and the warp-uniform exp skip of the 8^3
// kernels.
// ---------------------------------------------------------------------------

struct __align__(16) WarpStage4 {
    Rec rec[32];
    int32_t gid[32];
    int32_t pidx[32];  // deterministic backward: emission index of the pair
};

template <bool COMPAT, bool DET>
__device__ __forceinline__ int stage4(const RenderArgs& a, WarpStage4& S, int base, int cnt, int lane, int d0,
                                      int h0, int w0, const float ih[3]) {
    Rec r;
    int gid = 0;
    bool keep = false;
    if (lane < cnt) {
        gid = __ldg(a.pair_ids + base + lane);
        r = load_rec<COMPAT>(a, gid, ih);
        keep = true;
        if (a.cull) {
            float4 x;
            if (COMPAT) {
                const float qc[6] = {r.q00, r.q01x2, r.q02x2, r.q11, r.q12x2, r.q22};
                x = tight_extent(qc);
            } else {
                x = __ldg(a.ext + gid);
            }
            keep = __fsub_rn(r.c0, x.x) <= float(d0 + 3) && __fadd_rn(r.c0, x.x) >= float(d0) &&
                   __fsub_rn(r.c1, x.y) <= float(h0 + 3) && __fadd_rn(r.c1, x.y) >= float(h0) &&
                   __fsub_rn(r.c2, x.z) <= float(w0 + 3) && __fadd_rn(r.c2, x.z) >= float(w0);
        }
    }
    const unsigned kept = __ballot_sync(kFull, keep);
    int64_t e = 0;
    if (DET && lane < cnt) e = emission_index(a, gid, d0 >> 2, h0 >> 2, w0 >> 2);
    if (DET && lane < cnt && !keep) {  // dropped pair: its partial is zero
        float4* dst = reinterpret_cast<float4*>(a.partials + e * kMomStride);
        dst[0] = dst[1] = dst[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (keep) {
        const int pos = __popc(kept & ((1u << lane) - 1u));
        S.rec[pos] = r;
        S.gid[pos] = gid;
        if (DET) S.pidx[pos] = int32_t(e);
    }
    return __popc(kept);
}

template <bool COMPAT, bool PLANAR>
__global__ void __launch_bounds__(kThreads) k_forward4(const RenderArgs a) {
    __shared__ WarpStage4 stage[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t tile = int64_t(blockIdx.x) * kWarps + warp;
    if (tile >= a.ntiles) return;  // warp-uniform; no CTA barrier below
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    const int2 rg = a.ranges[tile];
    float ih[3];
    compat_ih<COMPAT>(a, ih);
    const int gd = d0 + (lane >> 3), gh = h0 + ((lane >> 1) & 3), gw = w0 + 2 * (lane & 1);
    const float ev0 = float(gd), ev1 = float(gh), ev2 = float(gw);
    float accR[2] = {0.f, 0.f}, accI[2] = {0.f, 0.f};
    WarpStage4& S = stage[warp];
    for (int base = rg.x; base < rg.y; base += 32) {
        const int kept = stage4<COMPAT, false>(a, S, base, min(32, rg.y - base), lane, d0, h0, w0, ih);
        __syncwarp();
        for (int j = 0; j < kept; ++j) {
            const Rec g = S.rec[j];
            const float e0 = __fsub_rn(ev0, g.c0), e1 = __fsub_rn(ev1, g.c1);
            const float e2a = __fsub_rn(ev2, g.c2), e2b = __fsub_rn(ev2 + 1.0f, g.c2);
            const float A = row_a(g, e0, e1), B = row_b(g, e0, e1);
            const float m0 = row_m(g.q22, A, B, e2a), m1 = row_m(g.q22, A, B, e2b);
            if (!__any_sync(kFull, m0 <= kCut || m1 <= kCut)) continue;
            if (m0 <= kCut) {
                const float wgt = ex2_approx(m0 * kNegHalfLog2e);
                accR[0] = fmaf(wgt, g.rho_r, accR[0]);
                accI[0] = fmaf(wgt, g.rho_i, accI[0]);
            }
            if (m1 <= kCut) {
                const float wgt = ex2_approx(m1 * kNegHalfLog2e);
                accR[1] = fmaf(wgt, g.rho_r, accR[1]);
                accI[1] = fmaf(wgt, g.rho_i, accI[1]);
            }
        }
        __syncwarp();
    }
    if (gd >= a.d || gh >= a.h) return;
    const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + gw;
    if (PLANAR) {
        for (int i = 0; i < 2; ++i)
            if (gw + i < a.w) {
                a.vol_r[flat + i] = accR[i];
                a.vol_i[flat + i] = accI[i];
            }
    } else if (gw + 1 < a.w && (a.w & 1) == 0) {
        reinterpret_cast<float4*>(a.vol)[flat >> 1] = make_float4(accR[0], accI[0], accR[1], accI[1]);
    } else {
        float2* out = reinterpret_cast<float2*>(a.vol) + flat;
        for (int i = 0; i < 2; ++i)
            if (gw + i < a.w) out[i] = make_float2(accR[i], accI[i]);
    }
}

template <bool COMPAT, bool DET>
__global__ void __launch_bounds__(kThreads) k_backward4(const RenderArgs a) {
    __shared__ WarpStage4 stage[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t tile = int64_t(blockIdx.x) * kWarps + warp;
    if (tile >= a.ntiles) return;  // warp-uniform; no CTA barrier below
    const int2 rg = a.ranges[tile];
    if (rg.x >= rg.y) return;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    float ih[3];
    compat_ih<COMPAT>(a, ih);
    const int gd = d0 + (lane >> 3), gh = h0 + ((lane >> 1) & 3), gw = w0 + 2 * (lane & 1);
    float gr[2] = {0.f, 0.f}, gi[2] = {0.f, 0.f};
    if (gd < a.d && gh < a.h) {
        const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + gw;
        for (int i = 0; i < 2; ++i)
            if (gw + i < a.w) {
                if (COMPAT) {
                    gr[i] = __ldg(a.gv_r + flat + i);
                    gi[i] = __ldg(a.gv_i + flat + i);
                } else {
                    const float2 x = __ldg(reinterpret_cast<const float2*>(a.gvol) + flat + i);
                    gr[i] = x.x;
                    gi[i] = x.y;
                }
            }
    }
    const float ev0 = float(gd), ev1 = float(gh), ev2 = float(gw);
    WarpStage4& S = stage[warp];
    for (int base = rg.x; base < rg.y; base += 32) {
        const int kept = stage4<COMPAT, DET>(a, S, base, min(32, rg.y - base), lane, d0, h0, w0, ih);
        __syncwarp();
        for (int j = 0; j < kept; ++j) {
            const Rec g = S.rec[j];
            const float e0 = __fsub_rn(ev0, g.c0), e1 = __fsub_rn(ev1, g.c1);
            const float e2v[2] = {__fsub_rn(ev2, g.c2), __fsub_rn(ev2 + 1.0f, g.c2)};
            const float A = row_a(g, e0, e1), B = row_b(g, e0, e1);
            const float m[2] = {row_m(g.q22, A, B, e2v[0]), row_m(g.q22, A, B, e2v[1])};
            if (!__any_sync(kFull, m[0] <= kCut || m[1] <= kCut)) {
                if (DET && lane == 0) {  // no included voxel here: the pair's partial is zero
                    float4* dst = reinterpret_cast<float4*>(a.partials + int64_t(S.pidx[j]) * kMomStride);
                    dst[0] = dst[1] = dst[2] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                continue;
            }
            const float hr = -0.5f * g.rho_r, hi = -0.5f * g.rho_i;
            float Dr = 0.f, Di = 0.f, R0 = 0.f, R1 = 0.f, R2 = 0.f;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (m[k] <= kCut) {
                    const float wgt = ex2_approx(m[k] * kNegHalfLog2e);
                    const float av = wgt * fmaf(hi, gi[k], hr * gr[k]);
                    Dr = fmaf(wgt, gr[k], Dr);
                    Di = fmaf(wgt, gi[k], Di);
                    R0 += av;
                    const float ae = av * e2v[k];
                    R1 += ae;
                    R2 = fmaf(ae, e2v[k], R2);
                }
            }
            float v[16];
            v[0] = Dr;
            v[1] = Di;
            v[2] = e0 * R0;
            v[3] = e1 * R0;
            v[4] = R1;
            v[5] = (e0 * e0) * R0;
            v[6] = e1 * v[2];
            v[7] = e0 * R1;
            v[8] = (e1 * e1) * R0;
            v[9] = e1 * R1;
            v[10] = R2;
            const int gid = S.gid[j];
            if (COMPAT) {
#pragma unroll
                for (int i = 11; i < 16; ++i) v[i] = 0.f;
                compat_emit(a, g, gid, warp_reduce_scatter16(v, lane), lane, ih);
            } else {
                v[11] = 0.f;
                const float tot = warp_reduce_scatter12(v, lane);
                const int mi = moment12(lane);
                if (!(lane & 1) && mi >= 0 && mi < kMom) {
                    if (DET) a.partials[int64_t(S.pidx[j]) * kMomStride + mi] = tot;
                    else atomicAdd(a.accum + int64_t(gid) * kMomStride + mi, tot);
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Generic tile edge: one voxel per thread, Gaussians staged per CTA.
// ---------------------------------------------------------------------------

template <bool COMPAT, bool PLANAR>
__global__ void __launch_bounds__(kThreads) k_forward_generic(const RenderArgs a) {
    __shared__ Rec srec[kThreads];
    const int64_t tile = blockIdx.x;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    const int2 rg = a.ranges[tile];
    const int ts = a.ts;
    const int nvox = ts * ts * ts;
    float ih[3];
    compat_ih<COMPAT>(a, ih);
    for (int c0 = 0; c0 < nvox; c0 += kThreads) {  // uniform trip count
        const int vid = c0 + threadIdx.x;
        const int ld = vid / (ts * ts), lh = (vid / ts) % ts, lw = vid % ts;
        const int gd = d0 + ld, gh = h0 + lh, gw = w0 + lw;
        const bool valid = vid < nvox && gd < a.d && gh < a.h && gw < a.w;
        const float v0 = float(gd), v1 = float(gh), v2 = float(gw);
        float ar = 0.f, ai = 0.f;
        for (int base = rg.x; base < rg.y; base += kThreads) {  // uniform trip count
            const int cnt = min(kThreads, rg.y - base);
            __syncthreads();
            if (threadIdx.x < cnt) srec[threadIdx.x] = load_rec<COMPAT>(a, __ldg(a.pair_ids + base + threadIdx.x), ih);
            __syncthreads();
            for (int j = 0; j < cnt; ++j) {
                const Rec g = srec[j];
                const float e0 = __fsub_rn(v0, g.c0), e1 = __fsub_rn(v1, g.c1), e2 = __fsub_rn(v2, g.c2);
                const float m = row_m(g.q22, row_a(g, e0, e1), row_b(g, e0, e1), e2);
                if (m <= kCut) {
                    const float wgt = ex2_approx(m * kNegHalfLog2e);
                    ar = fmaf(wgt, g.rho_r, ar);
                    ai = fmaf(wgt, g.rho_i, ai);
                }
            }
        }
        if (valid) {
            const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + gw;
            if (PLANAR) {
                a.vol_r[flat] = ar;
                a.vol_i[flat] = ai;
            } else {
                reinterpret_cast<float2*>(a.vol)[flat] = make_float2(ar, ai);
            }
        }
    }
}

template <bool COMPAT, bool DET>
__global__ void __launch_bounds__(kThreads) k_backward_generic(const RenderArgs a) {
    __shared__ Rec srec[32];
    __shared__ int sgid[32];
    __shared__ int64_t sidx[32];
    __shared__ float sred[kWarps][kMom];
    const int64_t tile = blockIdx.x;
    const int2 rg = a.ranges[tile];
    if (rg.x >= rg.y) return;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    const int ts = a.ts;
    const int nvox = ts * ts * ts;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float ih[3];
    compat_ih<COMPAT>(a, ih);
    for (int base = rg.x; base < rg.y; base += 32) {
        const int cnt = min(32, rg.y - base);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const int gid = __ldg(a.pair_ids + base + threadIdx.x);
            sgid[threadIdx.x] = gid;
            srec[threadIdx.x] = load_rec<COMPAT>(a, gid, ih);
            if (DET) sidx[threadIdx.x] = emission_index(a, gid, d0 / ts, h0 / ts, w0 / ts);
        }
        __syncthreads();
        for (int j = 0; j < cnt; ++j) {
            const Rec g = srec[j];
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.f;
            for (int vid = threadIdx.x; vid < nvox; vid += kThreads) {
                const int ld = vid / (ts * ts), lh = (vid / ts) % ts, lw = vid % ts;
                const int gd = d0 + ld, gh = h0 + lh, gw = w0 + lw;
                if (gd >= a.d || gh >= a.h || gw >= a.w) continue;
                const float e0 = __fsub_rn(float(gd), g.c0), e1 = __fsub_rn(float(gh), g.c1);
                const float e2 = __fsub_rn(float(gw), g.c2);
                const float m = row_m(g.q22, row_a(g, e0, e1), row_b(g, e0, e1), e2);
                if (!(m <= kCut)) continue;
                const int64_t flat = (int64_t(gd) * a.h + gh) * a.w + gw;
                float gr, gi;
                if (COMPAT) {
                    gr = __ldg(a.gv_r + flat);
                    gi = __ldg(a.gv_i + flat);
                } else {
                    const float2 x = __ldg(reinterpret_cast<const float2*>(a.gvol) + flat);
                    gr = x.x;
                    gi = x.y;
                }
                const float wgt = ex2_approx(m * kNegHalfLog2e);
                const float av = wgt * fmaf(-0.5f * g.rho_i, gi, (-0.5f * g.rho_r) * gr);
                v[0] = fmaf(wgt, gr, v[0]);
                v[1] = fmaf(wgt, gi, v[1]);
                v[2] = fmaf(av, e0, v[2]);
                v[3] = fmaf(av, e1, v[3]);
                v[4] = fmaf(av, e2, v[4]);
                v[5] = fmaf(av * e0, e0, v[5]);
                v[6] = fmaf(av * e0, e1, v[6]);
                v[7] = fmaf(av * e0, e2, v[7]);
                v[8] = fmaf(av * e1, e1, v[8]);
                v[9] = fmaf(av * e1, e2, v[9]);
                v[10] = fmaf(av * e2, e2, v[10]);
            }
            const float tot = warp_reduce_scatter16(v, lane);
            if (!(lane & 1) && (lane >> 1) < kMom) sred[warp][lane >> 1] = tot;
            __syncthreads();
            // warp 0 combines the four warps in a fixed order
            if (warp == 0) {
                float t = 0.f;
                if (lane < kMom) t = ((sred[0][lane] + sred[1][lane]) + sred[2][lane]) + sred[3][lane];
                // compat_emit expects moment i in lane 2i
                const float spread = __shfl_sync(kFull, t, lane >> 1);
                const int gid = sgid[j];
                if (COMPAT) {
                    compat_emit(a, g, gid, spread, lane, ih);
                } else if (DET) {
                    if (lane < kMom) a.partials[sidx[j] * kMomStride + lane] = t;
                } else {
                    if (lane < kMom) atomicAdd(a.accum + int64_t(gid) * kMomStride + lane, t);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Finalize: moments -> dL/d(positions, scales, rotations, density).
// Chain rule of tile_voxelizer.py:284-290 and :77-84 (the torch autograd
// tail of the reference), in FP32.
// ---------------------------------------------------------------------------

// Deterministic moments of Gaussian g, one warp: the Gaussian's per-pair
// partials sit contiguously at its emission indices, in tile raster order;
// lane l sums entries l, l + 32, ... and a fixed xor tree sums the lanes.
// The order depends only on the tile box, so the result is bitwise
// reproducible.  Writes the moments where the atomic backward accumulates
// them.
__device__ __forceinline__ void gather_det_warp(const RenderArgs& a, int64_t g, int lane) {
    float mo[kMom];
#pragma unroll
    for (int i = 0; i < kMom; ++i) mo[i] = 0.f;
    const int cnt = a.boxes[g].w;
    const int64_t first = a.offsets[g];
    for (int c = lane; c < cnt; c += 32) {
        const int64_t e = first + c;
        if (e >= a.capacity) break;  // pair capacity overflow (flagged): no such partial
        const float4* src = reinterpret_cast<const float4*>(a.partials + e * kMomStride);
        const float4 x = src[0], y = src[1], z = src[2];
        mo[0] += x.x; mo[1] += x.y; mo[2] += x.z; mo[3] += x.w;
        mo[4] += y.x; mo[5] += y.y; mo[6] += y.z; mo[7] += y.w;
        mo[8] += z.x; mo[9] += z.y; mo[10] += z.z;
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
        for (int i = 0; i < kMom; ++i) mo[i] += __shfl_xor_sync(0xffffffffu, mo[i], off);
    if (lane == 0) {
        float4* dst = reinterpret_cast<float4*>(a.accum + g * kMomStride);
        dst[0] = make_float4(mo[0], mo[1], mo[2], mo[3]);
        dst[1] = make_float4(mo[4], mo[5], mo[6], mo[7]);
        dst[2] = make_float4(mo[8], mo[9], mo[10], 0.f);
    }
}

// Chain rule of one Gaussian from its 11 moments (accum).  The moments are
// cleared once read: the preprocess clears them too, so the atomic backward
// always starts from zero without a memset of its own.
__device__ __forceinline__ void finalize_one(const RenderArgs& a, int64_t g) {
    const gsv_params& p = a.prm;
    const gsv_grads& out = a.grd;
    float mo[kMom];
#pragma unroll
    for (int i = 0; i < kMom; ++i) mo[i] = a.accum[g * kMomStride + i];
    {
        float4* acc4 = reinterpret_cast<float4*>(a.accum + g * kMomStride);
        acc4[0] = acc4[1] = acc4[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const Rec R = a.recs[g];
    // dL/dcenter_vox, then dcenter/dpositions = 0.5 * shape = hs   (:284).
    // The reference sums this over included pairs only: a Gaussian with none
    // (e.g. NaN coefficients) gets exactly 0, not 0 * NaN.
    const bool has_center = mo[2] != 0.f || mo[3] != 0.f || mo[4] != 0.f;
    const float dc0 = has_center ? -(2.0f * R.q00 * mo[2] + R.q01x2 * mo[3] + R.q02x2 * mo[4]) : 0.f;
    const float dc1 = has_center ? -(R.q01x2 * mo[2] + 2.0f * R.q11 * mo[3] + R.q12x2 * mo[4]) : 0.f;
    const float dc2 = has_center ? -(R.q02x2 * mo[2] + R.q12x2 * mo[3] + 2.0f * R.q22 * mo[4]) : 0.f;
    out.positions[g * 3 + 0] = dc0 * a.hs[0];
    out.positions[g * 3 + 1] = dc1 * a.hs[1];
    out.positions[g * 3 + 2] = dc2 * a.hs[2];
    out.density_r[g] = mo[0];
    out.density_i[g] = mo[1];
    // dL/dM (normalised units), symmetric.
    float G[9];
    G[0] = mo[5] * a.ih[0] * a.ih[0];
    G[1] = G[3] = mo[6] * a.ih[0] * a.ih[1];
    G[2] = G[6] = mo[7] * a.ih[0] * a.ih[2];
    G[4] = mo[8] * a.ih[1] * a.ih[1];
    G[5] = G[7] = mo[9] * a.ih[1] * a.ih[2];
    G[8] = mo[10] * a.ih[2] * a.ih[2];
    // Rebuild R(qn), si = 1/(s+1e-8) and T = R diag(si).
    float q[4], s[3];
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = p.rotations[g * 4 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = p.scales[g * 3 + k];
    const float nrm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const float den = nrm + 1e-8f;
    const float w = q[0] / den, x = q[1] / den, y = q[2] / den, z = q[3] / den;
    float r[9];
    r[0] = 1.f - 2.f * y * y - 2.f * z * z;
    r[1] = 2.f * x * y - 2.f * z * w;
    r[2] = 2.f * x * z + 2.f * y * w;
    r[3] = 2.f * x * y + 2.f * z * w;
    r[4] = 1.f - 2.f * x * x - 2.f * z * z;
    r[5] = 2.f * y * z - 2.f * x * w;
    r[6] = 2.f * x * z - 2.f * y * w;
    r[7] = 2.f * y * z + 2.f * x * w;
    r[8] = 1.f - 2.f * x * x - 2.f * y * y;
    float si[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) si[j] = 1.0f / (s[j] + 1e-8f);
    // dL/dT = (G + G^T) T = 2 G T
    float gr[9], gsi[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += G[i * 3 + k] * (r[k * 3 + j] * si[j]);
            const float gt = 2.0f * acc;
            gr[i * 3 + j] = gt * si[j];
            gsi[j] += gt * r[i * 3 + j];
        }
#pragma unroll
    for (int j = 0; j < 3; ++j) out.scales[g * 3 + j] = -gsi[j] * si[j] * si[j];
    float gn[4];
    gn[0] = 2.f * (-z * gr[1] + y * gr[2] + z * gr[3] - x * gr[5] - y * gr[6] + x * gr[7]);
    gn[1] = 2.f * (y * gr[1] + z * gr[2] + y * gr[3] - 2.f * x * gr[4] - w * gr[5] + z * gr[6] + w * gr[7] -
                   2.f * x * gr[8]);
    gn[2] = 2.f * (-2.f * y * gr[0] + x * gr[1] + w * gr[2] + x * gr[3] + z * gr[5] - w * gr[6] + z * gr[7] -
                   2.f * y * gr[8]);
    gn[3] = 2.f * (-2.f * z * gr[0] - w * gr[1] + x * gr[2] + w * gr[3] - 2.f * z * gr[4] + y * gr[5] +
                   x * gr[6] + y * gr[7]);
    const float dot = gn[0] * w + gn[1] * x + gn[2] * y + gn[3] * z;
    const float corr = nrm > 0.f ? dot / (nrm * den) : 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) out.rotations[g * 4 + k] = gn[k] / den - q[k] * corr;
}

__global__ void __launch_bounds__(256) k_finalize(const RenderArgs a) {
    const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= a.prm.n) return;
    finalize_one(a, g);
}

// One warp per Gaussian (deterministic backward).
__global__ void __launch_bounds__(256) k_gather_det(const RenderArgs a) {
    const int64_t g = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    if (g >= a.prm.n) return;  // warp-uniform
    gather_det_warp(a, g, threadIdx.x & 31);
}

// ---------------------------------------------------------------------------
// Batched persistent launches: many volumes, one launch.  The descriptor
// table (one RenderArgs per volume) and prefix sums of tiles, Gaussians and
// pair capacities live in device memory; CTAs pull global tile indices from
// an atomic counter until the work runs out.
// ---------------------------------------------------------------------------

struct BatchTable {
    RenderArgs* items;
    int64_t* tile_prefix;   // [count + 1]
    int64_t* gauss_prefix;  // [count + 1]
    int64_t* cap_prefix;    // [count + 1]
    unsigned long long* counters;  // [2]: forward, backward work counters
    int count;
    int det;
};

__device__ __forceinline__ int find_item(const int64_t* prefix, int count, int64_t x) {
    int lo = 0, hi = count;  // largest i with prefix[i] <= x
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kThreads) k_forward8_batched(const BatchTable t) {
    __shared__ __align__(16) unsigned char smem_raw[kFwdSmem];
    __shared__ long long s_next;
    const int64_t total = t.tile_prefix[t.count];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_next = (long long)atomicAdd(&t.counters[0], 1ull);
        __syncthreads();
        const int64_t gt = s_next;
        if (gt >= total) break;
        const int i = find_item(t.tile_prefix, t.count, gt);
        forward_tile<false, false, 2>(t.items[i], gt - t.tile_prefix[i], 0, smem_raw);
    }
}

template <bool DET>
__global__ void __launch_bounds__(kThreads, 6) k_backward8_batched(const BatchTable t) {
    __shared__ __align__(16) WarpStage stage[kWarps];
    __shared__ long long s_next;
    const int64_t total = t.tile_prefix[t.count];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_next = (long long)atomicAdd(&t.counters[1], 1ull);
        __syncthreads();
        const int64_t gt = s_next;
        if (gt >= total) break;
        const int i = find_item(t.tile_prefix, t.count, gt);
        backward_tile<false, DET, 2>(t.items[i], gt - t.tile_prefix[i], 0, stage, 0);
    }
}

__global__ void __launch_bounds__(256) k_finalize_batched(const BatchTable t) {
    const int64_t total = t.gauss_prefix[t.count];
    for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total;
         x += int64_t(gridDim.x) * blockDim.x) {
        const int i = find_item(t.gauss_prefix, t.count, x);
        finalize_one(t.items[i], x - t.gauss_prefix[i]);
    }
}

// One warp per Gaussian of every volume (deterministic backward).
__global__ void __launch_bounds__(256) k_gather_det_batched(const BatchTable t) {
    const int64_t total = t.gauss_prefix[t.count];
    const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t x = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; x < total; x += warps) {
        const int i = find_item(t.gauss_prefix, t.count, x);  // warp-uniform
        gather_det_warp(t.items[i], x - t.gauss_prefix[i], threadIdx.x & 31);
    }
}

// ---------------------------------------------------------------------------
// Work census of the tile-8 kernels (diagnostic, no gradients): per listed
// (tile, Gaussian) pair it replays the render kernels' decisions with their
// arithmetic -- the extent cull per 4x8x8 row slot, the row-form quadratic
// and the FP32 cutoff -- and counts
//   out[0]  included candidates (m <= 9, voxel inside the volume),
//   out[1]  candidates the kernels evaluate m for (voxels of kept slots),
//   out[2]  lanes issued by the per-column exp / FMA blocks (32 per column
//           of a kept slot in which some lane is inside the cutoff),
//   out[3]  kept slots without any included voxel.
// out[0] / out[2] is the lane efficiency of the exp / FMA blocks.  The
// inclusion count covers every listed slot, culled or not, so it also checks
// that the cull drops no included voxel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_count_work(const RenderArgs a, unsigned long long* out) {
    const int64_t tile = blockIdx.x;
    const int2 rg = a.ranges[tile];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int d0, h0, w0;
    decode_tile(a, tile, d0, h0, w0);
    unsigned long long c_inc = 0, c_eval = 0, c_lanes = 0, c_empty = 0;
    const float ev1 = float(h0 + (lane & 7));
    const bool h_ok = h0 + (lane & 7) < a.h;
    for (int p = rg.x + warp; p < rg.y; p += kWarps) {
        const int gid = __ldg(a.pair_ids + p);
        float ih[3];
        compat_ih<false>(a, ih);
        const Rec g = load_rec<false>(a, gid, ih);
        const float4 x = __ldg(a.ext + gid);
        const bool hw = __fsub_rn(g.c1, x.y) <= float(h0 + 7) && __fadd_rn(g.c1, x.y) >= float(h0) &&
                        __fsub_rn(g.c2, x.z) <= float(w0 + 7) && __fadd_rn(g.c2, x.z) >= float(w0);
        const float lo = __fsub_rn(g.c0, x.x), hi = __fadd_rn(g.c0, x.x);
        const float e1 = __fsub_rn(ev1, g.c1);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int ds = d0 + 4 * r;
            const bool kept = !a.cull || (hw && lo <= float(ds + 3) && hi >= float(ds));
            const int gd = ds + (lane >> 3);
            const float e0 = __fsub_rn(float(gd), g.c0);
            const float A = row_a(g, e0, e1), B = row_b(g, e0, e1);
            bool slot_any = false;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float m = row_m(g.q22, A, B, __fsub_rn(float(w0 + k), g.c2));
                const bool in = m <= kCut;
                c_inc += (in && gd < a.d && h_ok && w0 + k < a.w) ? 1 : 0;
                const bool col = __any_sync(kFull, in);
                slot_any |= col;
                if (kept && col && lane == 0) c_lanes += 32;
            }
            if (kept) {
                c_eval += 8;
                if (!slot_any && lane == 0) c_empty += 1;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c_inc += __shfl_xor_sync(kFull, c_inc, o);
        c_eval += __shfl_xor_sync(kFull, c_eval, o);
        c_lanes += __shfl_xor_sync(kFull, c_lanes, o);
        c_empty += __shfl_xor_sync(kFull, c_empty, o);
    }
    if (lane == 0) {
        atomicAdd(out, c_inc);
        atomicAdd(out + 1, c_eval);
        atomicAdd(out + 2, c_lanes);
        atomicAdd(out + 3, c_empty);
    }
}

int grid_for(int64_t items, int block) {
    int64_t g = (items + block - 1) / block;
    return int(g < 1 ? 1 : g);
}

template <typename T>
const T* cat(const void* base, size_t off) {
    return reinterpret_cast<const T*>(static_cast<const char*>(base) + off);
}
template <typename T>
T* mat(void* base, size_t off) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
}

void fill_shape(RenderArgs& a, gsv_shape s) {
    a.d = s.d; a.h = s.h; a.w = s.w; a.ts = s.tile_size;
    a.nth = (s.h + s.tile_size - 1) / s.tile_size;
    a.ntw = (s.w + s.tile_size - 1) / s.tile_size;
    a.ntiles = int64_t((s.d + s.tile_size - 1) / s.tile_size) * a.nth * a.ntw;
    a.chunk = 32;
    a.cull = 1;
    a.split = 1;
    const float sh[3] = {float(s.d), float(s.h), float(s.w)};
    for (int k = 0; k < 3; ++k) {
        a.hs[k] = sh[k] * 0.5f;
        a.ih[k] = 1.0f / a.hs[k];
    }
}

bool shape_ok(int32_t ts, int32_t d, int32_t h, int32_t w) {
    return ts > 0 && d > 0 && h > 0 && w > 0 && d < (1 << 24) && h < (1 << 24) && w < (1 << 24);
}

}  // namespace

extern "C" {

int gsv_forward(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs,
                int64_t capacity, float* volume, void* stream) {
    return gsv_forward_ex(shape, n, ws_gauss, ws_pairs, capacity, volume, nullptr, stream);
}

static bool tuning_ok(const gsv_tuning* t) {
    return !t || ((t->rows_per_lane == 1 || t->rows_per_lane == 2) && t->chunk >= 1 && t->chunk <= 32 &&
                  (t->split == 0 || t->split == 1 || t->split == 2 || t->split == 4));
}

int gsv_forward_ex(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs, int64_t capacity,
                   float* volume, const gsv_tuning* tuning, void* stream) {
    if (!tuning_ok(tuning)) return GSV_ERR_INVALID_ARGUMENT;
    GaussLayout G;
    PairLayout P;
    int64_t ntiles = 0;
    if (layout_for(shape, n, capacity, 0, &G, &P, &ntiles) != GSV_OK || !ws_gauss || !volume ||
        (capacity > 0 && !ws_pairs))
        return GSV_ERR_INVALID_ARGUMENT;
    if (ntiles > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RenderArgs a{};
    fill_shape(a, shape);
    a.recs = cat<Rec>(ws_gauss, G.rec);
    a.ext = cat<float4>(ws_gauss, G.ext);
    a.ranges = cat<int2>(ws_gauss, G.ranges);
    a.pair_ids = capacity > 0 ? cat<int32_t>(ws_pairs, P.vals_out) : nullptr;
    a.vol = volume;
    const int rpl = tuning ? tuning->rows_per_lane : 2;
    if (tuning) {
        a.chunk = tuning->chunk;
        a.cull = !(tuning->flags & GSV_TUNE_NO_CULL);
    }
    if (shape.tile_size == 8 && rpl == 2) k_forward8<false, false, 2><<<unsigned(ntiles), kThreads, 0, st>>>(a);
    else if (shape.tile_size == 8) k_forward8<false, false, 1><<<unsigned(2 * ntiles), kThreads, 0, st>>>(a);
    else if (shape.tile_size == 4)
        k_forward4<false, false><<<unsigned((ntiles + kWarps - 1) / kWarps), kThreads, 0, st>>>(a);
    else k_forward_generic<false, false><<<unsigned(ntiles), kThreads, 0, st>>>(a);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_backward(const gsv_params* p, gsv_shape shape, void* ws_gauss, void* ws_pairs,
                 int64_t capacity, const float* grad_volume, const gsv_grads* grads, int flags,
                 void* stream) {
    return gsv_backward_ex(p, shape, ws_gauss, ws_pairs, capacity, grad_volume, grads, flags, nullptr, stream);
}

int gsv_backward_ex(const gsv_params* p, gsv_shape shape, void* ws_gauss, void* ws_pairs, int64_t capacity,
                    const float* grad_volume, const gsv_grads* grads, int flags, const gsv_tuning* tuning,
                    void* stream) {
    if (!tuning_ok(tuning)) return GSV_ERR_INVALID_ARGUMENT;
    GaussLayout G;
    PairLayout P;
    int64_t ntiles = 0;
    const bool det = flags & GSV_BACKWARD_DETERMINISTIC;
    if (!p || !grads || layout_for(shape, p->n, capacity, flags, &G, &P, &ntiles) != GSV_OK || !ws_gauss ||
        !grad_volume || (capacity > 0 && !ws_pairs))
        return GSV_ERR_INVALID_ARGUMENT;
    const int64_t n = p->n;
    if (n == 0) return GSV_OK;
    if (!grads->positions || !grads->scales || !grads->rotations || !grads->density_r || !grads->density_i ||
        !p->scales || !p->rotations)
        return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RenderArgs a{};
    fill_shape(a, shape);
    a.recs = cat<Rec>(ws_gauss, G.rec);
    a.ext = cat<float4>(ws_gauss, G.ext);
    a.ranges = cat<int2>(ws_gauss, G.ranges);
    a.pair_ids = capacity > 0 ? cat<int32_t>(ws_pairs, P.vals_out) : nullptr;
    a.gvol = grad_volume;
    a.accum = mat<float>(ws_gauss, G.accum);
    a.partials = det ? mat<float>(ws_pairs, P.partials) : nullptr;
    a.offsets = cat<int64_t>(ws_gauss, G.offsets);
    a.boxes = cat<int4>(ws_gauss, G.box);
    a.capacity = capacity;
    // The atomic accumulators are zero here: the preprocess clears them and
    // k_finalize clears them again after reading.  The deterministic mode
    // writes every listed pair's partial and its gather overwrites them.
    if (tuning) {
        a.chunk = tuning->chunk;
        a.cull = !(tuning->flags & GSV_TUNE_NO_CULL);
        a.split = tuning->split > 1 ? tuning->split : 1;
    }
    if (ntiles * 2 * a.split > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    const int rpl = (tuning && !det) ? tuning->rows_per_lane : 2;  // deterministic: whole tiles
    const unsigned sp = unsigned(a.split);
    if (capacity > 0) {
        if (shape.tile_size == 8) {
            if (det) k_backward8<false, true, 2><<<unsigned(ntiles) * sp, kThreads, 0, st>>>(a);
            else if (rpl == 2) k_backward8<false, false, 2><<<unsigned(ntiles) * sp, kThreads, 0, st>>>(a);
            else k_backward8<false, false, 1><<<unsigned(2 * ntiles) * sp, kThreads, 0, st>>>(a);
        } else {
            const unsigned g4 = unsigned((ntiles + kWarps - 1) / kWarps);
            if (shape.tile_size == 4 && det) k_backward4<false, true><<<g4, kThreads, 0, st>>>(a);
            else if (shape.tile_size == 4) k_backward4<false, false><<<g4, kThreads, 0, st>>>(a);
            else if (det) k_backward_generic<false, true><<<unsigned(ntiles), kThreads, 0, st>>>(a);
            else k_backward_generic<false, false><<<unsigned(ntiles), kThreads, 0, st>>>(a);
        }
        GSV_LAUNCH_CHECK();
    }
    a.prm = *p;
    a.grd = *grads;
    if (det) {
        k_gather_det<<<grid_for(n * 32, 256), 256, 0, st>>>(a);
        GSV_LAUNCH_CHECK();
    }
    k_finalize<<<grid_for(n, 256), 256, 0, st>>>(a);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_count_work(gsv_shape shape, int64_t n, const void* ws_gauss, const void* ws_pairs, int64_t capacity,
                   const gsv_tuning* tuning, unsigned long long* out, void* stream) {
    if (!tuning_ok(tuning) || shape.tile_size != 8 || !out) return GSV_ERR_INVALID_ARGUMENT;
    GaussLayout G;
    PairLayout P;
    int64_t ntiles = 0;
    if (layout_for(shape, n, capacity, 0, &G, &P, &ntiles) != GSV_OK || !ws_gauss || (capacity > 0 && !ws_pairs))
        return GSV_ERR_INVALID_ARGUMENT;
    if (ntiles > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GSV_CUDA_TRY(cudaMemsetAsync(out, 0, 4 * sizeof(unsigned long long), st));
    if (capacity == 0 || n == 0) return GSV_OK;
    RenderArgs a{};
    fill_shape(a, shape);
    a.recs = cat<Rec>(ws_gauss, G.rec);
    a.ext = cat<float4>(ws_gauss, G.ext);
    a.ranges = cat<int2>(ws_gauss, G.ranges);
    a.pair_ids = cat<int32_t>(ws_pairs, P.vals_out);
    if (tuning) a.cull = !(tuning->flags & GSV_TUNE_NO_CULL);
    k_count_work<<<unsigned(ntiles), kThreads, 0, st>>>(a, out);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_tile_forward(const float* centers, const float* cov_inv, const float* density_r,
                     const float* density_i, const int32_t* tile_ranges, const int32_t* pair_ids,
                     const float* half_shape, int64_t n, int64_t num_tiles, int32_t tile_size,
                     int32_t d, int32_t h, int32_t w, float* vol_r, float* vol_i, void* stream) {
    if (!shape_ok(tile_size, d, h, w) || n < 0 || !tile_ranges || !half_shape || !vol_r || !vol_i)
        return GSV_ERR_INVALID_ARGUMENT;
    gsv_shape s{d, h, w, tile_size};
    RenderArgs a{};
    fill_shape(a, s);
    if (num_tiles != a.ntiles || num_tiles > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!centers || !cov_inv || !density_r || !density_i)) return GSV_ERR_INVALID_ARGUMENT;
    a.centers = centers;
    a.cov_inv = cov_inv;
    a.den_r = density_r;
    a.den_i = density_i;
    a.half_shape = half_shape;
    a.ranges = reinterpret_cast<const int2*>(tile_ranges);
    a.pair_ids = pair_ids;
    a.vol_r = vol_r;
    a.vol_i = vol_i;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (tile_size == 8) k_forward8<true, true, 2><<<unsigned(num_tiles), kThreads, 0, st>>>(a);
    else if (tile_size == 4)
        k_forward4<true, true><<<unsigned((num_tiles + kWarps - 1) / kWarps), kThreads, 0, st>>>(a);
    else k_forward_generic<true, true><<<unsigned(num_tiles), kThreads, 0, st>>>(a);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_tile_backward(const float* centers, const float* cov_inv, const float* density_r,
                      const float* density_i, const int32_t* tile_ranges, const int32_t* pair_ids,
                      const float* half_shape, const float* grad_vol_r, const float* grad_vol_i,
                      int64_t n, int64_t num_tiles, int32_t tile_size, int32_t d, int32_t h,
                      int32_t w, float* grad_centers, float* grad_cov_inv, float* grad_den_r,
                      float* grad_den_i, void* stream) {
    if (!shape_ok(tile_size, d, h, w) || n < 0 || !tile_ranges || !half_shape || !grad_vol_r ||
        !grad_vol_i)
        return GSV_ERR_INVALID_ARGUMENT;
    gsv_shape s{d, h, w, tile_size};
    RenderArgs a{};
    fill_shape(a, s);
    if (num_tiles != a.ntiles || num_tiles > int64_t(INT32_MAX)) return GSV_ERR_INVALID_ARGUMENT;
    if (n == 0) return GSV_OK;
    if (!centers || !cov_inv || !density_r || !density_i || !grad_centers || !grad_cov_inv ||
        !grad_den_r || !grad_den_i)
        return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GSV_CUDA_TRY(cudaMemsetAsync(grad_centers, 0, size_t(n) * 3 * sizeof(float), st));
    GSV_CUDA_TRY(cudaMemsetAsync(grad_cov_inv, 0, size_t(n) * 9 * sizeof(float), st));
    GSV_CUDA_TRY(cudaMemsetAsync(grad_den_r, 0, size_t(n) * sizeof(float), st));
    GSV_CUDA_TRY(cudaMemsetAsync(grad_den_i, 0, size_t(n) * sizeof(float), st));
    a.centers = centers;
    a.cov_inv = cov_inv;
    a.den_r = density_r;
    a.den_i = density_i;
    a.half_shape = half_shape;
    a.ranges = reinterpret_cast<const int2*>(tile_ranges);
    a.pair_ids = pair_ids;
    a.gv_r = grad_vol_r;
    a.gv_i = grad_vol_i;
    a.g_center = grad_centers;
    a.g_cov = grad_cov_inv;
    a.g_dr = grad_den_r;
    a.g_di = grad_den_i;
    if (tile_size == 8) k_backward8<true, false, 2><<<unsigned(num_tiles), kThreads, 0, st>>>(a);
    else if (tile_size == 4)
        k_backward4<true, false><<<unsigned((num_tiles + kWarps - 1) / kWarps), kThreads, 0, st>>>(a);
    else k_backward_generic<true, false><<<unsigned(num_tiles), kThreads, 0, st>>>(a);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

size_t gsv_batch_workspace_bytes(int count) {
    if (count <= 0 || count > (1 << 16)) return 0;
    return align_up(size_t(count) * sizeof(RenderArgs)) + 3 * align_up(size_t(count + 1) * sizeof(int64_t)) +
           align_up(2 * sizeof(unsigned long long));
}

int gsv_batch_setup(const gsv_batch_item* items, int count, int flags, void* ws_batch, size_t ws_bytes,
                    void* stream) {
    if (!items || count <= 0 || !ws_batch || ws_bytes < gsv_batch_workspace_bytes(count))
        return GSV_ERR_INVALID_ARGUMENT;
    const bool det = flags & GSV_BACKWARD_DETERMINISTIC;
    RenderArgs* host = new RenderArgs[count];
    int64_t* pre = new int64_t[3 * (count + 1)];
    int64_t *tp = pre, *gp = pre + count + 1, *cp = pre + 2 * (count + 1);
    tp[0] = gp[0] = cp[0] = 0;
    int rc = GSV_OK;
    for (int i = 0; i < count && rc == GSV_OK; ++i) {
        const gsv_batch_item& it = items[i];
        GaussLayout G;
        PairLayout P;
        int64_t ntiles = 0;
        if (it.shape.tile_size != 8 || layout_for(it.shape, it.params.n, it.capacity, flags, &G, &P, &ntiles) != GSV_OK ||
            !it.ws_gauss || (it.capacity > 0 && !it.ws_pairs)) {
            rc = GSV_ERR_INVALID_ARGUMENT;
            break;
        }
        RenderArgs a{};
        fill_shape(a, it.shape);
        a.recs = cat<Rec>(it.ws_gauss, G.rec);
        a.ext = cat<float4>(it.ws_gauss, G.ext);
        a.ranges = cat<int2>(it.ws_gauss, G.ranges);
        a.pair_ids = it.capacity > 0 ? cat<int32_t>(it.ws_pairs, P.vals_out) : nullptr;
        a.vol = it.volume;
        a.gvol = it.grad_volume;
        a.accum = mat<float>(const_cast<void*>(it.ws_gauss), G.accum);
        a.partials = det && it.capacity > 0 ? mat<float>(const_cast<void*>(it.ws_pairs), P.partials) : nullptr;
        a.prm = it.params;
        a.grd = it.grads;
        a.boxes = cat<int4>(it.ws_gauss, G.box);
        a.offsets = cat<int64_t>(it.ws_gauss, G.offsets);
        a.capacity = it.capacity;
        a.chunk = (it.chunk >= 1 && it.chunk <= 32) ? it.chunk : 32;
        host[i] = a;
        tp[i + 1] = tp[i] + ntiles;
        gp[i + 1] = gp[i] + it.params.n;
        cp[i + 1] = cp[i] + (det ? it.capacity : 0);
    }
    if (rc == GSV_OK) {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        char* base = static_cast<char*>(ws_batch);
        const size_t o_items = 0, o_pre = align_up(size_t(count) * sizeof(RenderArgs));
        cudaError_t e = cudaMemcpyAsync(base + o_items, host, size_t(count) * sizeof(RenderArgs),
                                        cudaMemcpyHostToDevice, st);
        for (int k = 0; k < 3 && e == cudaSuccess; ++k)
            e = cudaMemcpyAsync(base + o_pre + k * align_up(size_t(count + 1) * sizeof(int64_t)),
                                pre + k * (count + 1), size_t(count + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                                st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            gsv_detail_set_error(e, "gsv_batch_setup upload", __FILE__, __LINE__);
            rc = GSV_ERR_CUDA;
        }
    }
    delete[] host;
    delete[] pre;
    return rc;
}

namespace {
BatchTable batch_table(void* ws_batch, int count, int det) {
    BatchTable t{};
    char* base = static_cast<char*>(ws_batch);
    const size_t o_pre = align_up(size_t(count) * sizeof(RenderArgs));
    const size_t step = align_up(size_t(count + 1) * sizeof(int64_t));
    t.items = reinterpret_cast<RenderArgs*>(base);
    t.tile_prefix = reinterpret_cast<int64_t*>(base + o_pre);
    t.gauss_prefix = reinterpret_cast<int64_t*>(base + o_pre + step);
    t.cap_prefix = reinterpret_cast<int64_t*>(base + o_pre + 2 * step);
    t.counters = reinterpret_cast<unsigned long long*>(base + o_pre + 3 * step);
    t.count = count;
    t.det = det;
    return t;
}

// Persistent grid: every SM filled to the kernel's occupancy.
int persistent_grid(const void* kernel, int threads) {
    int dev = 0, sms = 148, per_sm = 4;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 4;
    return sms * per_sm;
}
}  // namespace

int gsv_forward_batched(void* ws_batch, int count, void* stream) {
    if (!ws_batch || count <= 0) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchTable t = batch_table(ws_batch, count, 0);
    GSV_CUDA_TRY(cudaMemsetAsync(t.counters, 0, 2 * sizeof(unsigned long long), st));
    k_forward8_batched<<<persistent_grid(reinterpret_cast<const void*>(k_forward8_batched), kThreads), kThreads, 0, st>>>(t);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

int gsv_backward_batched(void* ws_batch, int count, int flags, void* stream) {
    if (!ws_batch || count <= 0) return GSV_ERR_INVALID_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool det = flags & GSV_BACKWARD_DETERMINISTIC;
    BatchTable t = batch_table(ws_batch, count, det);
    GSV_CUDA_TRY(cudaMemsetAsync(t.counters, 0, 2 * sizeof(unsigned long long), st));
    // every volume's accumulators are zero: its preprocess cleared them and
    // k_finalize(_batched) clears them again after reading
    const int grid = persistent_grid(reinterpret_cast<const void*>(k_finalize_batched), 256);
    if (det) k_backward8_batched<true><<<persistent_grid(reinterpret_cast<const void*>(k_backward8_batched<true>), kThreads), kThreads, 0, st>>>(t);
    else k_backward8_batched<false><<<persistent_grid(reinterpret_cast<const void*>(k_backward8_batched<false>), kThreads), kThreads, 0, st>>>(t);
    GSV_LAUNCH_CHECK();
    if (det) {
        k_gather_det_batched<<<persistent_grid(reinterpret_cast<const void*>(k_gather_det_batched), 256), 256, 0,
                               st>>>(t);
        GSV_LAUNCH_CHECK();
    }
    k_finalize_batched<<<grid, 256, 0, st>>>(t);
    GSV_LAUNCH_CHECK();
    return GSV_OK;
}

}  // extern "C"
