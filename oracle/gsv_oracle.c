/*
 * gsv_oracle.c -- CPU oracle for the complex-Gaussian tile voxelizer.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (gs_tmi_b200/) links,
 * loads or calls this file; only tests/, the smoke check and bench.py's CPU
 * baseline leg do, as the checker.
 *
 * What it restates (paths are relative to the 3DGSMR project root,
 * V = 3DGS/3dgsVC):
 *   - preprocess           V/gaussian/tile_voxelizer.py:282-290, :77-84
 *   - tile binning         V/gaussian/tile_voxelizer.py:87-162
 *   - forward sum          V/gaussian/tile_voxelizer.py:210-244 and
 *                          V/gaussian/cuda_ext/tile_voxelize_cuda_kernel.cu:118-135
 *   - analytic backward    V/gaussian/cuda_ext/tile_voxelize_cuda_kernel.cu:233-252
 *                          plus the torch autograd chain through :282-290
 *
 * Precision contract:
 *   - The binning quantities (center_vox, radius_vox, the clamped voxel and
 *     tile boxes) are computed in FP32 in exactly the op order of
 *     tile_voxelizer.py:284-286 and :97-114, so tile lists are bit-exact with
 *     the reference.  Float->int conversion follows CUDA semantics
 *     (saturating, NaN -> 0), i.e. what the reference does on its GPU path.
 *   - The inclusion predicate "mahal <= 9" is evaluated in FP32 with the
 *     fixed op sequence the CUDA kernels use (quadratic form in voxel units,
 *     explicit fmaf), so kernel and oracle include exactly the same
 *     (voxel, Gaussian) pairs.
 *   - Everything else (centers, covariance inverse, distances, weights,
 *     sums, gradients, chain rule) is FP64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* FP32 helpers (compiled with -ffp-contract=off: no implicit FMA).     */
/* ------------------------------------------------------------------ */

/* CUDA float->int32 conversion: round toward zero, saturate, NaN -> 0. */
static int32_t f2i_sat(float x) {
    if (isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x < -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

static int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

/* torch max-reduction semantics: NaN propagates. */
static float nanmax3(float a, float b, float c) {
    if (isnan(a) || isnan(b) || isnan(c)) return NAN;
    float m = a > b ? a : b;
    return m > c ? m : c;
}

/*
 * FP32 quadratic-form coefficients of one Gaussian, in voxel units:
 *   m(e) = e^T Q e,  Q_ab = M_ab / (hs_a hs_b),  e = v - center_vox.
 * Stored as {q00, 2 q01, 2 q02, q11, 2 q12, q22}.
 * M = T T^T with T = R(q / (|q| + 1e-8)) diag(1 / (s + 1e-8))
 * (tile_voxelizer.py:77-84, :287-290).  Op order is the kernel's.
 */
static void rot_f32(const float* q, float* r) {
    float n2 = q[0] * q[0];
    n2 = n2 + q[1] * q[1];
    n2 = n2 + q[2] * q[2];
    n2 = n2 + q[3] * q[3];
    float den = sqrtf(n2) + 1e-8f;
    float w = q[0] / den, x = q[1] / den, y = q[2] / den, z = q[3] / den;
    float tx = 2.0f * x, ty = 2.0f * y, tz = 2.0f * z;
    r[0] = (1.0f - ty * y) - tz * z;
    r[1] = tx * y - tz * w;
    r[2] = tx * z + ty * w;
    r[3] = tx * y + tz * w;
    r[4] = (1.0f - tx * x) - tz * z;
    r[5] = ty * z - tx * w;
    r[6] = tx * z - ty * w;
    r[7] = ty * z + tx * w;
    r[8] = (1.0f - tx * x) - ty * y;
}

static void qcoef_f32(const float* s, const float* q, const float* ih, float* out) {
    float r[9];
    rot_f32(q, r);
    float si[3];
    for (int j = 0; j < 3; ++j) si[j] = 1.0f / (s[j] + 1e-8f);
    float t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = r[i * 3 + j] * si[j];
    static const int ia[6] = {0, 0, 0, 1, 1, 2};
    static const int ib[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) {
        const float* ta = &t[ia[k] * 3];
        const float* tb = &t[ib[k] * 3];
        float m = ta[0] * tb[0];
        m = m + ta[1] * tb[1];
        m = m + ta[2] * tb[2];
        float qv = (m * ih[ia[k]]) * ih[ib[k]];
        out[k] = (ia[k] == ib[k]) ? qv : 2.0f * qv;
    }
}

/* Same coefficients from an explicit 3x3 cov_inv in normalised units (the
 * reference extension's input, tile_voxelize_cuda.cpp:5-16); the matrix is
 * symmetrised as (M_ab + M_ba) * 0.5, exact for symmetric input. */
static void qcoef_from_covinv_f32(const float* m9, const float* ih, float* out) {
    static const int ia[6] = {0, 0, 0, 1, 1, 2};
    static const int ib[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < 6; ++k) {
        float m = (m9[ia[k] * 3 + ib[k]] + m9[ib[k] * 3 + ia[k]]) * 0.5f;
        float qv = (m * ih[ia[k]]) * ih[ib[k]];
        out[k] = (ia[k] == ib[k]) ? qv : 2.0f * qv;
    }
}

/* The FP32 inclusion test shared with the kernels. */
static int included_f32(const float* qc, float e0, float e1, float e2) {
    float u = fmaf(qc[1], e1, qc[0] * e0);
    float a = fmaf(u, e0, (qc[3] * e1) * e1);
    float b = fmaf(qc[4], e1, qc[2] * e0);
    float m = fmaf(fmaf(qc[5], e2, b), e2, a);
    return m <= 9.0f;
}

/* ------------------------------------------------------------------ */
/* The reference's own FP32 op order for the inclusion test.           */
/*                                                                      */
/* tile_voxelize_cuda_kernel.cu:118-130 evaluates, per voxel v and      */
/* Gaussian (c, M):                                                     */
/*   dx = (v0 - c0) / hs0  (dy, dz alike)                               */
/*   md_a = M_a0 dx + M_a1 dy + M_a2 dz                                 */
/*   mahal = dx md_0 + dy md_1 + dz md_2,  included iff mahal <= 9      */
/* in FP32 with nvcc's default contraction of a left-to-right sum of    */
/* products: the first product rounded, each later one fused,           */
/* fma(x2, y2, fma(x1, y1, x0 * y0)).  The extension is built with       */
/* --use_fast_math (tile_voxelizer.py:58-66), whose division is          */
/* approximate; ORC_PRED_REFERENCE_RCP models it as a product with the   */
/* correctly rounded reciprocal.  Both agree with IEEE division when hs  */
/* is a power of two.  M is the FP32 cov_inv the reference passes in:   */
/* in the compat layout the caller's array; in the params layout         */
/* T T^T with T = R(q) diag(1 / (s + 1e-8)) (tile_voxelizer.py:287-290)  */
/* accumulated with FMAs, as a batched GEMM does.                        */
/* ------------------------------------------------------------------ */

enum { ORC_PRED_ROWFORM = 0, ORC_PRED_REFERENCE = 1, ORC_PRED_REFERENCE_RCP = 2 };
static int g_pred = ORC_PRED_ROWFORM;

/* Selects the inclusion test of orc_forward / orc_backward; returns the
 * previous mode.  Not thread-safe: oracle.py serialises its callers. */
ORC_EXPORT int orc_set_predicate(int mode) {
    int old = g_pred;
    g_pred = (mode == ORC_PRED_REFERENCE || mode == ORC_PRED_REFERENCE_RCP) ? mode : ORC_PRED_ROWFORM;
    return old;
}

static void refcov_f32(const float* s, const float* q, float* m9) {
    float r[9], si[3], t[9];
    rot_f32(q, r);
    for (int j = 0; j < 3; ++j) si[j] = 1.0f / (s[j] + 1e-8f);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = r[i * 3 + j] * si[j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const float* ta = &t[i * 3];
            const float* tb = &t[j * 3];
            m9[i * 3 + j] = fmaf(ta[2], tb[2], fmaf(ta[1], tb[1], ta[0] * tb[0]));
        }
}

static int included_ref_f32(int mode, const float* c, const float* m, const float* hs, float v0, float v1,
                            float v2) {
    float dx, dy, dz;
    if (mode == ORC_PRED_REFERENCE_RCP) {
        dx = (v0 - c[0]) * (1.0f / hs[0]);
        dy = (v1 - c[1]) * (1.0f / hs[1]);
        dz = (v2 - c[2]) * (1.0f / hs[2]);
    } else {
        dx = (v0 - c[0]) / hs[0];
        dy = (v1 - c[1]) / hs[1];
        dz = (v2 - c[2]) / hs[2];
    }
    float md0 = fmaf(m[2], dz, fmaf(m[1], dy, m[0] * dx));
    float md1 = fmaf(m[5], dz, fmaf(m[4], dy, m[3] * dx));
    float md2 = fmaf(m[8], dz, fmaf(m[7], dy, m[6] * dx));
    float mahal = fmaf(dz, md2, fmaf(dy, md1, dx * md0));
    return mahal <= 9.0f;
}

/* ------------------------------------------------------------------ */
/* Preprocess (FP32, bit-exact with the reference where it matters).  */
/* ------------------------------------------------------------------ */

ORC_EXPORT void orc_preprocess_f32(const float* pos, const float* scl, const float* rot, int64_t n,
                                   int32_t d, int32_t h, int32_t w, float* center, float* radius,
                                   float* qcoef) {
    const float shape[3] = {(float)d, (float)h, (float)w};
    float hs[3], ih[3];
    for (int a = 0; a < 3; ++a) {
        hs[a] = shape[a] * 0.5f;
        ih[a] = 1.0f / hs[a];
    }
    for (int64_t g = 0; g < n; ++g) {
        float sv[3];
        for (int a = 0; a < 3; ++a) {
            /* center_vox = (positions + 1.0) * 0.5 * shape - 0.5  (:284) */
            float c = pos[g * 3 + a] + 1.0f;
            c = c * 0.5f;
            c = c * shape[a];
            c = c - 0.5f;
            if (center) center[g * 3 + a] = c;
            sv[a] = scl[g * 3 + a] * hs[a]; /* scale_vox (:285) */
        }
        if (radius) radius[g] = nanmax3(sv[0], sv[1], sv[2]) * 3.0f; /* (:286) */
        if (qcoef) qcoef_f32(&scl[g * 3], &rot[g * 4], ih, &qcoef[g * 6]);
    }
}

ORC_EXPORT void orc_qcoef_from_covinv_f32(const float* cov_inv, const float* half_shape, int64_t n,
                                          float* qcoef) {
    float ih[3];
    for (int a = 0; a < 3; ++a) ih[a] = 1.0f / half_shape[a];
    for (int64_t g = 0; g < n; ++g) qcoef_from_covinv_f32(&cov_inv[g * 9], ih, &qcoef[g * 6]);
}

/* ------------------------------------------------------------------ */
/* Binning  (tile_voxelizer.py:87-162).                                */
/* box[g*6..]: tile_min d,h,w then tile count per axis d,h,w.          */
/* Returns total pairs, or -1 if some Gaussian has an empty box        */
/* (negative radius), which the reference cannot handle either.        */
/* ------------------------------------------------------------------ */

ORC_EXPORT int64_t orc_count_pairs(const float* center, const float* radius, int64_t n, int32_t d,
                                   int32_t h, int32_t w, int32_t ts, int32_t* counts, int32_t* box) {
    const int32_t size[3] = {d, h, w};
    const int32_t nt[3] = {(d + ts - 1) / ts, (h + ts - 1) / ts, (w + ts - 1) / ts};
    int64_t total = 0;
    for (int64_t g = 0; g < n; ++g) {
        int64_t cnt = 1;
        for (int a = 0; a < 3; ++a) {
            float c = center[g * 3 + a];
            float r = radius[g];
            int32_t lo = clampi(f2i_sat(floorf(c - r)), 0, size[a] - 1);
            int32_t hi = clampi(f2i_sat(ceilf(c + r)), 0, size[a] - 1);
            int32_t tlo = clampi(lo / ts, 0, nt[a] - 1);
            int32_t thi = clampi(hi / ts, 0, nt[a] - 1);
            int32_t na = thi - tlo + 1;
            if (na <= 0) return -1;
            box[g * 6 + a] = tlo;
            box[g * 6 + 3 + a] = na;
            cnt *= na;
        }
        counts[g] = (int32_t)cnt;
        total += cnt;
    }
    return total;
}

ORC_EXPORT void orc_fill_pairs(const int32_t* counts, const int32_t* box, int64_t n, int32_t d,
                               int32_t h, int32_t w, int32_t ts, int32_t* tile_ranges,
                               int32_t* pair_ids) {
    (void)counts;
    const int32_t nth = (h + ts - 1) / ts, ntw = (w + ts - 1) / ts;
    const int64_t ntiles = (int64_t)((d + ts - 1) / ts) * nth * ntw;
    int64_t* hist = (int64_t*)calloc((size_t)ntiles + 1, sizeof(int64_t));
    for (int64_t g = 0; g < n; ++g) {
        const int32_t* b = &box[g * 6];
        for (int32_t i = 0; i < b[3]; ++i)
            for (int32_t j = 0; j < b[4]; ++j)
                for (int32_t k = 0; k < b[5]; ++k)
                    hist[((int64_t)(b[0] + i) * nth + (b[1] + j)) * ntw + (b[2] + k)]++;
    }
    int64_t* cursor = (int64_t*)malloc(((size_t)ntiles + 1) * sizeof(int64_t));
    int64_t acc = 0;
    for (int64_t t = 0; t < ntiles; ++t) {
        cursor[t] = acc;
        if (hist[t] > 0) {
            tile_ranges[t * 2] = (int32_t)acc;
            tile_ranges[t * 2 + 1] = (int32_t)(acc + hist[t]);
        } else {
            tile_ranges[t * 2] = 0; /* empty tiles keep (0, 0): tile_voxelizer.py:151 */
            tile_ranges[t * 2 + 1] = 0;
        }
        acc += hist[t];
    }
    /* Ascending gid within each tile: the order a stable sort of the
     * Gaussian-major generation order (:126-149) produces. */
    for (int64_t g = 0; g < n; ++g) {
        const int32_t* b = &box[g * 6];
        for (int32_t i = 0; i < b[3]; ++i)
            for (int32_t j = 0; j < b[4]; ++j)
                for (int32_t k = 0; k < b[5]; ++k) {
                    int64_t t = ((int64_t)(b[0] + i) * nth + (b[1] + j)) * ntw + (b[2] + k);
                    pair_ids[cursor[t]++] = (int32_t)g;
                }
    }
    free(cursor);
    free(hist);
}

/* ------------------------------------------------------------------ */
/* FP64 Gaussian state.                                                 */
/* ------------------------------------------------------------------ */

typedef struct {
    double c[3];    /* center in voxels */
    double m[9];    /* cov_inv, normalised units */
    double r[9];    /* rotation of the normalised quaternion */
    double qn[4];   /* normalised quaternion */
    double qnorm;   /* |q| */
    double si[3];   /* 1 / (s + 1e-8) */
    double rho[2];
} g64_t;

static void gauss64(const double* p, const double* s, const double* q, double dr, double di,
                    const double* shape, g64_t* g) {
    for (int a = 0; a < 3; ++a) g->c[a] = (p[a] + 1.0) * 0.5 * shape[a] - 0.5;
    double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    g->qnorm = n;
    for (int k = 0; k < 4; ++k) g->qn[k] = q[k] / (n + 1e-8);
    double w = g->qn[0], x = g->qn[1], y = g->qn[2], z = g->qn[3];
    double* r = g->r;
    r[0] = 1 - 2 * y * y - 2 * z * z;
    r[1] = 2 * x * y - 2 * z * w;
    r[2] = 2 * x * z + 2 * y * w;
    r[3] = 2 * x * y + 2 * z * w;
    r[4] = 1 - 2 * x * x - 2 * z * z;
    r[5] = 2 * y * z - 2 * x * w;
    r[6] = 2 * x * z - 2 * y * w;
    r[7] = 2 * y * z + 2 * x * w;
    r[8] = 1 - 2 * x * x - 2 * y * y;
    for (int j = 0; j < 3; ++j) g->si[j] = 1.0 / (s[j] + 1e-8);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double acc = 0;
            for (int j = 0; j < 3; ++j) acc += r[a * 3 + j] * r[b * 3 + j] * g->si[j] * g->si[j];
            g->m[a * 3 + b] = acc;
        }
    g->rho[0] = dr;
    g->rho[1] = di;
}

/* Per-Gaussian accumulated gradient moments in normalised coordinates:
 * [0..1] dL/drho (re, im), [2..4] dL/dcenter_vox, [5..13] dL/dcov_inv (3x3). */
#define NMOM 14

/* Chain rule from (dL/dcenter_vox, dL/dcov_inv) to the raw parameters,
 * mirroring the autograd graph of tile_voxelizer.py:284-290 and :77-84. */
static void chain_rule64(const g64_t* g, const double* mom, const double* shape, double* gp,
                         double* gs, double* gq) {
    for (int a = 0; a < 3; ++a) gp[a] = mom[2 + a] * 0.5 * shape[a];
    const double* G = &mom[5];
    /* T = R diag(si); M = T T^T; dL/dT = (G + G^T) T */
    double t[9], gt[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = g->r[i * 3 + j] * g->si[j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int k = 0; k < 3; ++k) acc += (G[i * 3 + k] + G[k * 3 + i]) * t[k * 3 + j];
            gt[i * 3 + j] = acc;
        }
    double gr[9];
    for (int j = 0; j < 3; ++j) {
        double gsi = 0;
        for (int i = 0; i < 3; ++i) {
            gr[i * 3 + j] = gt[i * 3 + j] * g->si[j];
            gsi += gt[i * 3 + j] * g->r[i * 3 + j];
        }
        gs[j] = -gsi * g->si[j] * g->si[j];
    }
    double w = g->qn[0], x = g->qn[1], y = g->qn[2], z = g->qn[3];
    double gn[4];
    gn[0] = 2 * (-z * gr[1] + y * gr[2] + z * gr[3] - x * gr[5] - y * gr[6] + x * gr[7]);
    gn[1] = 2 * (y * gr[1] + z * gr[2] + y * gr[3] - 2 * x * gr[4] - w * gr[5] + z * gr[6] + w * gr[7] -
                 2 * x * gr[8]);
    gn[2] = 2 * (-2 * y * gr[0] + x * gr[1] + w * gr[2] + x * gr[3] + z * gr[5] - w * gr[6] + z * gr[7] -
                 2 * y * gr[8]);
    gn[3] = 2 * (-2 * z * gr[0] - w * gr[1] + x * gr[2] + w * gr[3] - 2 * z * gr[4] + y * gr[5] + x * gr[6] +
                 y * gr[7]);
    /* qn = q / (|q| + eps) */
    double n = g->qnorm, den = n + 1e-8;
    double dot = gn[0] * g->qn[0] + gn[1] * g->qn[1] + gn[2] * g->qn[2] + gn[3] * g->qn[3];
    for (int k = 0; k < 4; ++k) {
        double qk = g->qn[k] * den; /* raw q */
        double term = (n > 0) ? qk * dot * den / (n * den * den) : 0.0;
        gq[k] = gn[k] / den - term;
    }
}

/* ------------------------------------------------------------------ */
/* Forward / backward.                                                  */
/*                                                                      */
/* Two parameterisations:                                               */
/*   - "params": raw (positions, scales, rotations, density) as the     */
/*     TileVoxelizer module takes them;                                 */
/*   - "compat": (center_vox, cov_inv, density, half_shape) as the      */
/*     reference extension takes them (tile_voxelize_cuda.cpp:5-31).    */
/* The predicate always comes from the FP32 inputs; the FP64 arithmetic */
/* comes from the optional FP64 overrides (used for finite differences) */
/* or from the FP32 inputs widened.                                     */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t d, h, w, ts, nth, ntw;
    int64_t ntiles;
} shape_t;

static shape_t mkshape(int32_t d, int32_t h, int32_t w, int32_t ts) {
    shape_t s;
    s.d = d; s.h = h; s.w = w; s.ts = ts;
    s.nth = (h + ts - 1) / ts;
    s.ntw = (w + ts - 1) / ts;
    s.ntiles = (int64_t)((d + ts - 1) / ts) * s.nth * s.ntw;
    return s;
}

/* Build FP32 predicate state (centers + Q coefficients) and FP64 state. */
static void build_state(int compat, int64_t n, const shape_t* sh, const float* a32, const float* b32,
                        const float* c32, const float* dr32, const float* di32, const float* hs32,
                        const double* a64, const double* b64, const double* c64, const double* dr64,
                        const double* di64, float* cen32, float* qc32, g64_t* g64) {
    const double shape[3] = {sh->d, sh->h, sh->w};
    if (!compat) {
        orc_preprocess_f32(a32, b32, c32, n, sh->d, sh->h, sh->w, cen32, NULL, qc32);
        for (int64_t g = 0; g < n; ++g) {
            double p[3], s[3], q[4];
            for (int k = 0; k < 3; ++k) {
                p[k] = a64 ? a64[g * 3 + k] : (double)a32[g * 3 + k];
                s[k] = b64 ? b64[g * 3 + k] : (double)b32[g * 3 + k];
            }
            for (int k = 0; k < 4; ++k) q[k] = c64 ? c64[g * 4 + k] : (double)c32[g * 4 + k];
            gauss64(p, s, q, dr64 ? dr64[g] : dr32[g], di64 ? di64[g] : di32[g], shape, &g64[g]);
        }
    } else {
        /* a = center_vox [n,3], b = cov_inv [n,9] */
        memcpy(cen32, a32, (size_t)n * 3 * sizeof(float));
        orc_qcoef_from_covinv_f32(b32, hs32, n, qc32);
        for (int64_t g = 0; g < n; ++g) {
            memset(&g64[g], 0, sizeof(g64_t));
            for (int k = 0; k < 3; ++k) g64[g].c[k] = a64 ? a64[g * 3 + k] : (double)a32[g * 3 + k];
            for (int k = 0; k < 9; ++k) g64[g].m[k] = b64 ? b64[g * 9 + k] : (double)b32[g * 9 + k];
            g64[g].rho[0] = dr64 ? dr64[g] : dr32[g];
            g64[g].rho[1] = di64 ? di64[g] : di32[g];
        }
    }
}

/* FP32 inputs of one inclusion test, in either op order. */
typedef struct {
    int mode;           /* ORC_PRED_* */
    const float* cen;   /* [n,3] center_vox */
    const float* qc;    /* [n,6] row-form coefficients (ORC_PRED_ROWFORM) */
    const float* m9;    /* [n,9] FP32 cov_inv (reference op orders) */
    float hs[3];        /* FP32 half shape (reference op orders) */
} pred_t;

/* m9 (may be NULL when mode is the row form): the reference's FP32 cov_inv. */
static void build_pred(int mode, int compat, int64_t n, const shape_t* sh, const float* b32,
                       const float* c32, const float* hs32, const float* cen32, const float* qc32,
                       float* m9, pred_t* P) {
    P->mode = mode;
    P->cen = cen32;
    P->qc = qc32;
    P->m9 = NULL;
    if (compat) {
        for (int a = 0; a < 3; ++a) P->hs[a] = hs32[a];
    } else {
        P->hs[0] = (float)sh->d * 0.5f;
        P->hs[1] = (float)sh->h * 0.5f;
        P->hs[2] = (float)sh->w * 0.5f;
    }
    if (mode == ORC_PRED_ROWFORM) return;
    if (compat) {
        P->m9 = b32;
    } else {
        for (int64_t g = 0; g < n; ++g) refcov_f32(&b32[g * 3], &c32[g * 4], &m9[g * 9]);
        P->m9 = m9;
    }
}

static int pred_incl(const pred_t* P, int32_t g, int32_t i, int32_t j, int32_t k) {
    const float* c = &P->cen[(int64_t)g * 3];
    if (P->mode == ORC_PRED_ROWFORM)
        return included_f32(&P->qc[(int64_t)g * 6], (float)i - c[0], (float)j - c[1], (float)k - c[2]);
    return included_ref_f32(P->mode, c, &P->m9[(int64_t)g * 9], P->hs, (float)i, (float)j, (float)k);
}

static void tile_origin(const shape_t* sh, int64_t t, int32_t* o) {
    int64_t per = (int64_t)sh->nth * sh->ntw;
    int32_t td = (int32_t)(t / per);
    int64_t rem = t % per;
    o[0] = td * sh->ts;
    o[1] = (int32_t)(rem / sh->ntw) * sh->ts;
    o[2] = (int32_t)(rem % sh->ntw) * sh->ts;
}

/* Evaluate one (voxel, Gaussian) pair in FP64: returns the weight, stores
 * normalised d and M d.  hs is the FP64 half shape. */
static double eval64(const g64_t* g, const double* v, const double* hs, double* dn, double* md) {
    for (int a = 0; a < 3; ++a) dn[a] = (v[a] - g->c[a]) / hs[a];
    double m = 0;
    for (int a = 0; a < 3; ++a) {
        md[a] = g->m[a * 3 + 0] * dn[0] + g->m[a * 3 + 1] * dn[1] + g->m[a * 3 + 2] * dn[2];
        m += dn[a] * md[a];
    }
    return exp(-0.5 * m);
}

static void half_shape64(int compat, const shape_t* sh, const float* hs32, double* hs) {
    if (compat) {
        for (int a = 0; a < 3; ++a) hs[a] = hs32[a];
    } else {
        hs[0] = sh->d * 0.5; hs[1] = sh->h * 0.5; hs[2] = sh->w * 0.5;
    }
}

/* vol: interleaved (re, im) FP64, length 2*d*h*w.
 * stats (may be NULL): [0] candidate evaluations, [1] included pairs. */
ORC_EXPORT int orc_forward(int compat, const float* a32, const float* b32, const float* c32,
                           const float* dr32, const float* di32, const float* hs32, const double* a64,
                           const double* b64, const double* c64, const double* dr64,
                           const double* di64, int64_t n, int32_t d, int32_t h, int32_t w, int32_t ts,
                           const int32_t* tile_ranges, const int32_t* pair_ids, double* vol,
                           int64_t* stats) {
    shape_t sh = mkshape(d, h, w, ts);
    float* cen32 = (float*)malloc((size_t)(n ? n : 1) * 3 * sizeof(float));
    float* qc32 = (float*)malloc((size_t)(n ? n : 1) * 6 * sizeof(float));
    g64_t* g64 = (g64_t*)malloc((size_t)(n ? n : 1) * sizeof(g64_t));
    build_state(compat, n, &sh, a32, b32, c32, dr32, di32, hs32, a64, b64, c64, dr64, di64, cen32, qc32,
                g64);
    float* m9 = (g_pred != ORC_PRED_ROWFORM && !compat) ? (float*)malloc((size_t)(n ? n : 1) * 9 * sizeof(float))
                                                         : NULL;
    pred_t P;
    build_pred(g_pred, compat, n, &sh, b32, c32, hs32, cen32, qc32, m9, &P);
    double hs[3];
    half_shape64(compat, &sh, hs32, hs);
    memset(vol, 0, (size_t)d * h * w * 2 * sizeof(double));
    int64_t cand = 0, incl = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : cand, incl)
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t s0 = tile_ranges[t * 2], s1 = tile_ranges[t * 2 + 1];
        if (s0 >= s1) continue;
        int32_t o[3];
        tile_origin(&sh, t, o);
        for (int32_t i = o[0]; i < o[0] + ts && i < d; ++i)
            for (int32_t j = o[1]; j < o[1] + ts && j < h; ++j)
                for (int32_t k = o[2]; k < o[2] + ts && k < w; ++k) {
                    double acc_r = 0, acc_i = 0;
                    double v[3] = {i, j, k};
                    for (int32_t p = s0; p < s1; ++p) {
                        int32_t g = pair_ids[p];
                        ++cand;
                        if (!pred_incl(&P, g, i, j, k)) continue;
                        ++incl;
                        double dn[3], md[3];
                        double wgt = eval64(&g64[g], v, hs, dn, md);
                        acc_r += wgt * g64[g].rho[0];
                        acc_i += wgt * g64[g].rho[1];
                    }
                    int64_t f = ((int64_t)i * h + j) * w + k;
                    vol[f * 2] = acc_r;
                    vol[f * 2 + 1] = acc_i;
                }
    }
    if (stats) {
        stats[0] = cand;
        stats[1] = incl;
    }
    free(m9);
    free(cen32);
    free(qc32);
    free(g64);
    return 0;
}

/* Backward.  grad_vol: interleaved (re, im) FP64 upstream gradient.
 * params mode outputs: o1 = d/dpositions [n,3], o2 = d/dscales [n,3],
 *                      o3 = d/drotations [n,4], o4/o5 = d/ddensity re/im [n].
 * compat mode outputs: o1 = d/dcenter_vox [n,3], o2 = d/dcov_inv [n,9],
 *                      o3 unused, o4/o5 = d/ddensity re/im [n].
 * Per-(tile, Gaussian) partial moments are formed in parallel and summed
 * per Gaussian in list order, so the result is deterministic. */
ORC_EXPORT int orc_backward(int compat, const float* a32, const float* b32, const float* c32,
                            const float* dr32, const float* di32, const float* hs32, const double* a64,
                            const double* b64, const double* c64, const double* dr64,
                            const double* di64, int64_t n, int32_t d, int32_t h, int32_t w,
                            int32_t ts, const int32_t* tile_ranges, const int32_t* pair_ids,
                            int64_t n_pairs, const double* grad_vol, double* o1, double* o2,
                            double* o3, double* o4, double* o5) {
    shape_t sh = mkshape(d, h, w, ts);
    int64_t nn = n ? n : 1;
    float* cen32 = (float*)malloc((size_t)nn * 3 * sizeof(float));
    float* qc32 = (float*)malloc((size_t)nn * 6 * sizeof(float));
    g64_t* g64 = (g64_t*)malloc((size_t)nn * sizeof(g64_t));
    build_state(compat, n, &sh, a32, b32, c32, dr32, di32, hs32, a64, b64, c64, dr64, di64, cen32, qc32,
                g64);
    float* m9 = (g_pred != ORC_PRED_ROWFORM && !compat) ? (float*)malloc((size_t)nn * 9 * sizeof(float)) : NULL;
    pred_t P;
    build_pred(g_pred, compat, n, &sh, b32, c32, hs32, cen32, qc32, m9, &P);
    double hs[3];
    half_shape64(compat, &sh, hs32, hs);
    double* part = (double*)calloc((size_t)(n_pairs ? n_pairs : 1) * NMOM, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t s0 = tile_ranges[t * 2], s1 = tile_ranges[t * 2 + 1];
        if (s0 >= s1) continue;
        int32_t o[3];
        tile_origin(&sh, t, o);
        for (int32_t p = s0; p < s1; ++p) {
            int32_t g = pair_ids[p];
            const g64_t* G = &g64[g];
            double* mo = &part[(int64_t)p * NMOM];
            for (int32_t i = o[0]; i < o[0] + ts && i < d; ++i)
                for (int32_t j = o[1]; j < o[1] + ts && j < h; ++j)
                    for (int32_t k = o[2]; k < o[2] + ts && k < w; ++k) {
                        if (!pred_incl(&P, g, i, j, k)) continue;
                        int64_t f = ((int64_t)i * h + j) * w + k;
                        double gvr = grad_vol[f * 2], gvi = grad_vol[f * 2 + 1];
                        double v[3] = {i, j, k}, dn[3], md[3];
                        double wgt = eval64(G, v, hs, dn, md);
                        double dldm = -0.5 * wgt * (G->rho[0] * gvr + G->rho[1] * gvi);
                        mo[0] += wgt * gvr;
                        mo[1] += wgt * gvi;
                        for (int a = 0; a < 3; ++a) mo[2 + a] += dldm * (-2.0 * md[a] / hs[a]);
                        for (int a = 0; a < 3; ++a)
                            for (int b = 0; b < 3; ++b) mo[5 + a * 3 + b] += dldm * dn[a] * dn[b];
                    }
        }
    }
    double* tot = (double*)calloc((size_t)nn * NMOM, sizeof(double));
    for (int64_t p = 0; p < n_pairs; ++p) {
        int32_t g = pair_ids[p];
        for (int k = 0; k < NMOM; ++k) tot[(int64_t)g * NMOM + k] += part[p * NMOM + k];
    }
    const double shape[3] = {d, h, w};
    for (int64_t g = 0; g < n; ++g) {
        const double* mo = &tot[g * NMOM];
        o4[g] = mo[0];
        o5[g] = mo[1];
        if (compat) {
            for (int a = 0; a < 3; ++a) o1[g * 3 + a] = mo[2 + a];
            for (int k = 0; k < 9; ++k) o2[g * 9 + k] = mo[5 + k];
        } else {
            chain_rule64(&g64[g], mo, shape, &o1[g * 3], &o2[g * 3], &o3[g * 4]);
        }
    }
    free(tot);
    free(part);
    free(m9);
    free(cen32);
    free(qc32);
    free(g64);
    return 0;
}

/* Candidate-evaluation count E = sum over tiles of |list| * |voxels in tile|. */
ORC_EXPORT int64_t orc_candidate_evals(const int32_t* tile_ranges, int32_t d, int32_t h, int32_t w,
                                       int32_t ts) {
    shape_t sh = mkshape(d, h, w, ts);
    int64_t e = 0;
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t o[3];
        tile_origin(&sh, t, o);
        int64_t nv = (int64_t)((o[0] + ts < d ? ts : d - o[0])) * (o[1] + ts < h ? ts : h - o[1]) *
                     (o[2] + ts < w ? ts : w - o[2]);
        e += (int64_t)(tile_ranges[t * 2 + 1] - tile_ranges[t * 2]) * nv;
    }
    return e;
}

/* Listed (voxel, Gaussian) candidates on which two inclusion tests
 * disagree.  out[0]: included by both, out[1]: by mode_a only, out[2]: by
 * mode_b only, out[3]: candidates.  vflags (may be NULL, [d*h*w]): set to 1
 * at every voxel with a disagreement.  Inputs as orc_forward's FP32 ones. */
ORC_EXPORT int orc_predicate_flips(int compat, const float* a32, const float* b32, const float* c32,
                                   const float* hs32, int64_t n, int32_t d, int32_t h, int32_t w, int32_t ts,
                                   const int32_t* tile_ranges, const int32_t* pair_ids, int mode_a, int mode_b,
                                   int64_t* out, uint8_t* vflags) {
    shape_t sh = mkshape(d, h, w, ts);
    int64_t nn = n ? n : 1;
    float* cen32 = (float*)malloc((size_t)nn * 3 * sizeof(float));
    float* qc32 = (float*)malloc((size_t)nn * 6 * sizeof(float));
    float* m9 = compat ? NULL : (float*)malloc((size_t)nn * 9 * sizeof(float));
    if (compat) {
        memcpy(cen32, a32, (size_t)n * 3 * sizeof(float));
        orc_qcoef_from_covinv_f32(b32, hs32, n, qc32);
    } else {
        orc_preprocess_f32(a32, b32, c32, n, d, h, w, cen32, NULL, qc32);
    }
    pred_t PA, PB;
    build_pred(mode_a, compat, n, &sh, b32, c32, hs32, cen32, qc32, m9, &PA);
    build_pred(mode_b, compat, n, &sh, b32, c32, hs32, cen32, qc32, m9, &PB);
    if (vflags) memset(vflags, 0, (size_t)d * h * w);
    int64_t both = 0, a_only = 0, b_only = 0, cand = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : both, a_only, b_only, cand)
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t s0 = tile_ranges[t * 2], s1 = tile_ranges[t * 2 + 1];
        if (s0 >= s1) continue;
        int32_t o[3];
        tile_origin(&sh, t, o);
        for (int32_t i = o[0]; i < o[0] + ts && i < d; ++i)
            for (int32_t j = o[1]; j < o[1] + ts && j < h; ++j)
                for (int32_t k = o[2]; k < o[2] + ts && k < w; ++k) {
                    int flip = 0;
                    for (int32_t p = s0; p < s1; ++p) {
                        int32_t g = pair_ids[p];
                        int ia = pred_incl(&PA, g, i, j, k), ib = pred_incl(&PB, g, i, j, k);
                        ++cand;
                        both += ia && ib;
                        a_only += ia && !ib;
                        b_only += ib && !ia;
                        flip |= ia != ib;
                    }
                    if (flip && vflags) vflags[((int64_t)i * h + j) * w + k] = 1;
                }
    }
    out[0] = both;
    out[1] = a_only;
    out[2] = b_only;
    out[3] = cand;
    free(m9);
    free(cen32);
    free(qc32);
    return 0;
}

ORC_EXPORT int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Voxels that have some listed Gaussian with |m64 - 9| <= tol.  An FP32
 * evaluation in another op order (the reference's torch path, its CUDA
 * kernel with fast math) may decide such a pair differently from the shared
 * predicate; comparisons against those implementations exclude these
 * voxels and count them.  Returns the number of flagged voxels. */
ORC_EXPORT int64_t orc_boundary_voxels(const float* pos, const float* scl, const float* rot, int64_t n,
                                       int32_t d, int32_t h, int32_t w, int32_t ts,
                                       const int32_t* tile_ranges, const int32_t* pair_ids, double tol,
                                       uint8_t* flags) {
    shape_t sh = mkshape(d, h, w, ts);
    int64_t nn = n ? n : 1;
    g64_t* g64 = (g64_t*)malloc((size_t)nn * sizeof(g64_t));
    const double shape[3] = {d, h, w};
    for (int64_t g = 0; g < n; ++g) {
        double p[3], s[3], q[4];
        for (int k = 0; k < 3; ++k) {
            p[k] = pos[g * 3 + k];
            s[k] = scl[g * 3 + k];
        }
        for (int k = 0; k < 4; ++k) q[k] = rot[g * 4 + k];
        gauss64(p, s, q, 0, 0, shape, &g64[g]);
    }
    const double hs[3] = {d * 0.5, h * 0.5, w * 0.5};
    memset(flags, 0, (size_t)d * h * w);
    int64_t count = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : count)
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t s0 = tile_ranges[t * 2], s1 = tile_ranges[t * 2 + 1];
        if (s0 >= s1) continue;
        int32_t o[3];
        tile_origin(&sh, t, o);
        for (int32_t i = o[0]; i < o[0] + ts && i < d; ++i)
            for (int32_t j = o[1]; j < o[1] + ts && j < h; ++j)
                for (int32_t k = o[2]; k < o[2] + ts && k < w; ++k) {
                    double v[3] = {i, j, k}, dn[3], md[3];
                    int hit = 0;
                    for (int32_t p = s0; p < s1 && !hit; ++p) {
                        double wgt = eval64(&g64[pair_ids[p]], v, hs, dn, md);
                        double m = -2.0 * log(wgt);
                        if (fabs(m - 9.0) <= tol) hit = 1;
                    }
                    if (hit) {
                        flags[((int64_t)i * h + j) * w + k] = 1;
                        ++count;
                    }
                }
    }
    free(g64);
    return count;
}

/* Extent cull of the tile-8 render kernels, checked against the shared FP32
 * predicate.  The kernels skip a Gaussian (or a 4x8x8 row slot of it) whose
 * conservative tight extent ext_a -- 3 sqrt(S_aa (1 + 1e-4 K)) + 0.01 voxel,
 * S = Q^-1 and K = max_a Q_aa S_aa, infinite when Q is not positive
 * definite or K > 1e4, computed in FP64 and rounded up to FP32 -- misses
 * the slot: c_a - ext_a > hi_a or c_a + ext_a < lo_a, in FP32.  Restated
 * here from that rule.  For every listed (voxel, Gaussian) pair that the
 * FP32 predicate includes, the voxel's slot must pass that test; returns the
 * number of included pairs that would be culled (must be 0) and, in
 * stats[0..2], the pairs listed, the pairs kept and the row slots kept
 * (slots: the two 4x8x8 halves of each 8^3 tile). */
static float ext_f32_up(double v) {
    float f = (float)v;
    if ((double)f < v) f = nextafterf(f, INFINITY);
    return f;
}

static void extent_of(const float* qc, float ext[3]) {
    double q00 = qc[0], q01 = 0.5 * (double)qc[1], q02 = 0.5 * (double)qc[2];
    double q11 = qc[3], q12 = 0.5 * (double)qc[4], q22 = qc[5];
    double c00 = q11 * q22 - q12 * q12, c11 = q00 * q22 - q02 * q02, c22 = q00 * q11 - q01 * q01;
    double c01 = q02 * q12 - q01 * q22, c02 = q01 * q12 - q02 * q11;
    double det = q00 * c00 + q01 * c01 + q02 * c02;
    ext[0] = ext[1] = ext[2] = INFINITY;
    if (!(q00 > 0.0 && c22 > 0.0 && det > 0.0 && c00 > 0.0 && c11 > 0.0)) return;
    double s[3] = {c00 / det, c11 / det, c22 / det};
    double k = fmax(fmax(q00 * s[0], q11 * s[1]), q22 * s[2]);
    if (!(k <= 1e4)) return;
    double f = 9.0 * (1.0 + 1e-4 * k);
    for (int a = 0; a < 3; ++a) ext[a] = ext_f32_up(sqrt(f * s[a]) + 0.01);
}

static int slot_live(const float* c, const float* ext, const int32_t lo[3], const int32_t hi[3]) {
    for (int a = 0; a < 3; ++a) {
        float l = c[a] - ext[a], u = c[a] + ext[a];
        if (!(l <= (float)hi[a] && u >= (float)lo[a])) return 0;
    }
    return 1;
}

ORC_EXPORT int64_t orc_extent_check(const float* pos, const float* scl, const float* rot, int64_t n,
                                    int32_t d, int32_t h, int32_t w, const int32_t* tile_ranges,
                                    const int32_t* pair_ids, int64_t* stats) {
    const int32_t ts = 8;
    shape_t sh = mkshape(d, h, w, ts);
    int64_t nn = n ? n : 1;
    float* cen = (float*)malloc((size_t)nn * 3 * sizeof(float));
    float* qc = (float*)malloc((size_t)nn * 6 * sizeof(float));
    float* ext = (float*)malloc((size_t)nn * 3 * sizeof(float));
    orc_preprocess_f32(pos, scl, rot, n, d, h, w, cen, NULL, qc);
    for (int64_t g = 0; g < n; ++g) extent_of(&qc[g * 6], &ext[g * 3]);
    int64_t bad = 0, listed = 0, kept = 0, slots = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad, listed, kept, slots)
    for (int64_t t = 0; t < sh.ntiles; ++t) {
        int32_t s0 = tile_ranges[t * 2], s1 = tile_ranges[t * 2 + 1];
        int32_t o[3];
        tile_origin(&sh, t, o);
        for (int32_t p = s0; p < s1; ++p) {
            const int32_t g = pair_ids[p];
            const float* c = &cen[g * 3];
            int any = 0;
            for (int half = 0; half < 2; ++half) {
                int32_t lo[3] = {o[0] + 4 * half, o[1], o[2]};
                int32_t hi[3] = {o[0] + 4 * half + 3, o[1] + 7, o[2] + 7};
                int live = slot_live(c, &ext[g * 3], lo, hi);
                any |= live;
                slots += live;
                for (int32_t i = lo[0]; i <= hi[0] && i < d; ++i)
                    for (int32_t j = lo[1]; j <= hi[1] && j < h; ++j)
                        for (int32_t k = lo[2]; k <= hi[2] && k < w; ++k) {
                            float e0 = (float)i - c[0], e1 = (float)j - c[1], e2 = (float)k - c[2];
                            if (included_f32(&qc[g * 6], e0, e1, e2) && !live) ++bad;
                        }
            }
            ++listed;
            kept += any;
        }
    }
    free(cen);
    free(qc);
    free(ext);
    if (stats) {
        stats[0] = listed;
        stats[1] = kept;
        stats[2] = slots;
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* Variable-density Poisson-disc k-space mask                           */
/* ------------------------------------------------------------------ */

/* Python slice bounds [start, stop) of `start:stop` on an axis of size n
 * (negative indices count from the end; both clipped to [0, n]). */
static void py_slice(int64_t start, int64_t stop, int64_t n, int64_t* lo, int64_t* hi) {
    if (start < 0) start += n;
    if (stop < 0) stop += n;
    if (start < 0) start = 0;
    if (stop < 0) stop = 0;
    if (start > n) start = n;
    if (stop > n) stop = n;
    *lo = start;
    *hi = stop > start ? stop : start;
}

/* V/data/mask_generator.py:241-390 (_generate_poisson_mask_heuristic):
 * the calibration square set first, then one pass of dart throwing over the
 * pixels in `order` (the reference's np.random.permutation): a pixel is
 * taken unless it is already set or an already taken pixel lies at squared
 * distance < radius^2 (radius = the reference's r_grid = 0.6 / sqrt(pdf)),
 * until `target` pixels are set.  Sequential, as the reference; returns the
 * number of pixels set. */
ORC_EXPORT int64_t orc_poisson_mask(const double* radius, const int32_t* order, int32_t ny, int32_t nz,
                                    int32_t calib, int64_t target, int8_t* mask) {
    const int64_t n = (int64_t)ny * nz;
    memset(mask, 0, (size_t)n);
    const int64_t cy = ny / 2, cz = nz / 2, h = calib / 2;
    int64_t y0, y1, z0, z1;
    py_slice(cy - h, cy + h, ny, &y0, &y1);
    py_slice(cz - h, cz + h, nz, &z0, &z1);
    int64_t count = 0;
    for (int64_t y = y0; y < y1; ++y)
        for (int64_t z = z0; z < z1; ++z) {
            mask[y * nz + z] = 1;
            ++count;
        }
    if (count >= target) return count;
    for (int64_t i = 0; i < n; ++i) {
        if (count >= target) break;
        const int64_t c = order[i];
        const int64_t y = c / nz, z = c % nz;
        if (mask[c]) continue;
        const double r = radius[c];
        const int64_t ir = (int64_t)ceil(r);
        const int64_t ya = y - ir > 0 ? y - ir : 0, yb = y + ir + 1 < ny ? y + ir + 1 : ny;
        const int64_t za = z - ir > 0 ? z - ir : 0, zb = z + ir + 1 < nz ? z + ir + 1 : nz;
        const double r2 = r * r;
        int clash = 0;
        for (int64_t py = ya; py < yb && !clash; ++py)
            for (int64_t pz = za; pz < zb; ++pz) {
                if (!mask[py * nz + pz]) continue;
                const double d2 = (double)((py - y) * (py - y) + (pz - z) * (pz - z));
                if (d2 < r2) {
                    clash = 1;
                    break;
                }
            }
        if (clash) continue;
        mask[c] = 1;
        ++count;
    }
    return count;
}
