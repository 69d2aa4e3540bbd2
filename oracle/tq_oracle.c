/*
 * tq_oracle.c -- plain-C restatement of TurboQuant's encode-and-scan path.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU checker; see tq_oracle.h).  Compiled with
 * -ffp-contract=off and without fast-math: every fmaf() below is an FMA the
 * reference's pinned build performs, every other operation rounds on its own.
 */
#include "tq_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_SQRT1_2
#define M_SQRT1_2 0.70710678118654752440
#endif
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct tqo_space {
    size_t dim, D, packed_bytes, code_size;
    int bits, num_levels, num_boundaries;
    float scale, wht_scale;
    float *centroids, *boundaries, *rot_signs, *qjl_signs;
};

/* The constants the reference's build folded (space_turbo_quant.h:348, 357-359):
 *   `norm > 1e-10f` is evaluated as `norm_sq > fl(1e-10f * 1e-10f)`,
 *   the floored sigma is 1e-10f and its inverse is fl(1 / 1e-10f). */
static float f32_from_bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
#define NORMSQ_FLOOR f32_from_bits(0x1E3CE509u)   /* fl(1e-10f * 1e-10f) */
#define SIGMA_FLOOR f32_from_bits(0x2EDBE6FFu)    /* 1e-10f */
#define INV_SIGMA_FLOOR f32_from_bits(0x501502F9u) /* fl(1.0f / 1e-10f) */

/* ---- splitmix64 + sign vectors: turbo_quant.h:27-39, 74-86 ---------------- */
static uint64_t splitmix64_next(uint64_t *state) {
    uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void tqo_signs(size_t d, uint64_t seed, float *out) {
    uint64_t state = seed;
    for (size_t i = 0; i < d; ++i)
        out[i] = (splitmix64_next(&state) & 1u) ? 1.0f : -1.0f;
}

/* ---- Lloyd-Max for N(0,1): space_turbo_quant.h:76-131 --------------------- */
static double lm_phi(double x) { return exp(-0.5 * x * x) / sqrt(2.0 * M_PI); }
static double lm_Phi(double x) { return 0.5 * erfc(-x * M_SQRT1_2); }
static double lm_cond_mean(double a, double b) {
    double denom = lm_Phi(b) - lm_Phi(a);
    if (denom < 1e-15) return 0.5 * (a + b);
    return (lm_phi(a) - lm_phi(b)) / denom;
}

void tqo_lloyd_max(int bits, float *centroids, float *boundaries) {
    const int levels = 1 << bits;
    const int half = levels / 2;
    double *pos_c = (double *)malloc(sizeof(double) * (size_t)half);
    double *pos_b = (double *)malloc(sizeof(double) * (size_t)(half > 1 ? half - 1 : 1));
    double *new_c = (double *)malloc(sizeof(double) * (size_t)half);
    for (int i = 0; i < half; ++i) pos_c[i] = (i + 0.5) * 3.5 / half;
    for (int iter = 0; iter < 1000; ++iter) {
        for (int i = 0; i < half - 1; ++i) pos_b[i] = 0.5 * (pos_c[i] + pos_c[i + 1]);
        double max_delta = 0.0;
        for (int i = 0; i < half; ++i) {
            double lo = (i == 0) ? 0.0 : pos_b[i - 1];
            double hi = (i == half - 1) ? 1e10 : pos_b[i];
            new_c[i] = lm_cond_mean(lo, hi);
            double dlt = fabs(new_c[i] - pos_c[i]);
            if (dlt > max_delta) max_delta = dlt;
        }
        memcpy(pos_c, new_c, sizeof(double) * (size_t)half);
        if (max_delta < 1e-12) break;
    }
    for (int i = 0; i < half; ++i) {
        centroids[half + i] = (float)pos_c[i];
        centroids[half - 1 - i] = -(float)pos_c[i];
    }
    boundaries[half - 1] = 0.0f;
    for (int i = 0; i < half - 1; ++i) {
        double b = 0.5 * (pos_c[i] + pos_c[i + 1]);
        boundaries[half + i] = (float)b;
        boundaries[half - 2 - i] = -(float)b;
    }
    free(pos_c); free(pos_b); free(new_c);
}

/* ---- geometry: space_turbo_quant.h:233-238, 258-266; turbo_quant.h:177-184 */
size_t tqo_padded_dim(size_t dim) {
    size_t d = dim < 4 ? 4 : dim, p = 1;
    while (p < d) p <<= 1;
    return p;
}
size_t tqo_packed_bytes(size_t D, int bits) { return bits <= 4 ? (D + 1) / 2 : D; }
size_t tqo_code_size(size_t D, int bits) { return tqo_packed_bytes(D, bits) + 12; }

tqo_space *tqo_create(size_t dim, int bits, uint64_t rot_seed, uint64_t qjl_seed) {
    if (dim < 1 || bits < 2 || bits > 9) return NULL;
    tqo_space *sp = (tqo_space *)calloc(1, sizeof(tqo_space));
    sp->dim = dim;
    sp->D = tqo_padded_dim(dim);
    sp->bits = bits;
    sp->packed_bytes = tqo_packed_bytes(sp->D, bits);
    sp->code_size = sp->packed_bytes + 12;
    sp->num_levels = 1 << (bits - 1);
    sp->num_boundaries = sp->num_levels - 1;
    /* space_turbo_quant.h:265-266: sqrt(float(pi)/2) / sqrt(float(D)) */
    sp->scale = sqrtf((float)M_PI / 2.0f) / sqrtf((float)sp->D);
    /* turbo_quant.h:69 */
    sp->wht_scale = 1.0f / sqrtf((float)sp->D);
    sp->centroids = (float *)malloc(sizeof(float) * (size_t)sp->num_levels);
    sp->boundaries = (float *)malloc(sizeof(float) * (size_t)(sp->num_boundaries + 1));
    tqo_lloyd_max(bits - 1, sp->centroids, sp->boundaries);
    sp->rot_signs = (float *)malloc(sizeof(float) * sp->D);
    sp->qjl_signs = (float *)malloc(sizeof(float) * sp->D);
    tqo_signs(sp->D, rot_seed, sp->rot_signs);
    tqo_signs(sp->D, qjl_seed, sp->qjl_signs);
    return sp;
}

void tqo_destroy(tqo_space *sp) {
    if (!sp) return;
    free(sp->centroids); free(sp->boundaries); free(sp->rot_signs); free(sp->qjl_signs);
    free(sp);
}
size_t tqo_space_padded_dim(const tqo_space *sp) { return sp->D; }
size_t tqo_space_code_size(const tqo_space *sp) { return sp->code_size; }
float tqo_space_scale(const tqo_space *sp) { return sp->scale; }
const float *tqo_space_centroids(const tqo_space *sp) { return sp->centroids; }
const float *tqo_space_boundaries(const tqo_space *sp) { return sp->boundaries; }
const float *tqo_space_rot_signs(const tqo_space *sp) { return sp->rot_signs; }
const float *tqo_space_qjl_signs(const tqo_space *sp) { return sp->qjl_signs; }

/* ---- the pinned build's sum-of-squares tree --------------------------------
 * Main loop: 8 lanes, lane k accumulates acc[k] = acc[k] + x[i]*x[i] for
 * i = k mod 8 in increasing i (multiply and add round separately).  Then
 * t[k] = acc[k] + acc[k+4] (k < 4) and s = (t0 + t2) + (t1 + t3).
 * If 4..7 elements remain: t[k] = fma(x, x, t[k]) on the next 4 elements and
 * s = (t0 + t2) + (t1 + t3) again (t starts at zero when n < 8).
 * The last n mod 4 elements: s = fma(x, x, s) in order.                      */
float tqo_sq_reduce(const float *x, size_t n) {
    float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float s = 0.0f;
    size_t base = 0;
    if (n >= 8) {
        float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        size_t n8 = n & ~(size_t)7;
        for (size_t i = 0; i < n8; i += 8)
            for (int k = 0; k < 8; ++k) {
                float p = x[i + k] * x[i + k];
                acc[k] = acc[k] + p;
            }
        for (int k = 0; k < 4; ++k) t[k] = acc[k] + acc[k + 4];
        s = (t[0] + t[2]) + (t[1] + t[3]);
        base = n8;
    }
    size_t r = n - base;
    if (r >= 4) {
        for (int k = 0; k < 4; ++k) t[k] = fmaf(x[base + k], x[base + k], t[k]);
        s = (t[0] + t[2]) + (t[1] + t[3]);
        base += 4;
        r -= 4;
    }
    for (size_t j = 0; j < r; ++j) s = fmaf(x[base + j], x[base + j], s);
    return s;
}

/* ---- randomized Hadamard: turbo_quant.h:46-72, 89-99 ----------------------- */
static void rht(float *v, const float *signs, size_t D, float wht_scale) {
    for (size_t i = 0; i < D; ++i) v[i] = v[i] * signs[i];
    for (size_t step = 1; step < D; step <<= 1)
        for (size_t i = 0; i < D; i += step << 1)
            for (size_t j = 0; j < step; ++j) {
                float a = v[i + j], b = v[i + step + j];
                v[i + j] = a + b;
                v[i + step + j] = a - b;
            }
    for (size_t i = 0; i < D; ++i) v[i] = v[i] * wht_scale;
}

/* quantize: space_turbo_quant.h:332-337 (strict `>` count, uint8 result) */
static uint8_t quantize(const tqo_space *sp, float v) {
    uint8_t idx = 0;
    for (int j = 0; j < sp->num_boundaries; ++j) idx = (uint8_t)(idx + (v > sp->boundaries[j]));
    return idx;
}

/* encodeVector: space_turbo_quant.h:339-396 */
static void encode_one(const tqo_space *sp, const float *raw, uint8_t *out,
                       float *rot, float *res, uint8_t *idx) {
    const size_t dim = sp->dim, D = sp->D;
    float norm_sq = tqo_sq_reduce(raw, dim);
    float norm = sqrtf(norm_sq);
    float inv_norm = (norm_sq > NORMSQ_FLOOR) ? 1.0f / norm : 0.0f;
    for (size_t i = 0; i < D; ++i) rot[i] = 0.0f;
    for (size_t i = 0; i < dim; ++i) rot[i] = raw[i] * inv_norm;
    rht(rot, sp->rot_signs, D, sp->wht_scale);

    float var = tqo_sq_reduce(rot, D);
    float sigma = sqrtf(var / (float)D);
    float inv_sigma;
    if (SIGMA_FLOOR > sigma) {
        sigma = SIGMA_FLOOR;
        inv_sigma = INV_SIGMA_FLOOR;
    } else {
        inv_sigma = 1.0f / sigma;
    }
    for (size_t i = 0; i < D; ++i) {
        float normalized = rot[i] * inv_sigma;
        idx[i] = quantize(sp, normalized);
        res[i] = fmaf(-sp->centroids[idx[i]], sigma, rot[i]); /* contracted */
    }
    float gamma = sqrtf(tqo_sq_reduce(res, D));
    rht(res, sp->qjl_signs, D, sp->wht_scale);

    if (sp->bits <= 4) {
        memset(out, 0, sp->packed_bytes);
        for (size_t i = 0; i < D; ++i) {
            uint8_t unit = (uint8_t)((idx[i] << 1) | (res[i] >= 0.0f ? 1u : 0u));
            if ((i & 1) == 0) out[i >> 1] = unit;
            else out[i >> 1] = (uint8_t)(out[i >> 1] | (unit << 4));
        }
    } else {
        for (size_t i = 0; i < D; ++i)
            out[i] = (uint8_t)((idx[i] << 1) | (res[i] >= 0.0f ? 1u : 0u));
    }
    float meta[3] = {norm, gamma, sigma};
    memcpy(out + sp->packed_bytes, meta, 12);
}

void tqo_encode_batch(const tqo_space *sp, const float *X, size_t n, uint8_t *out,
                      int num_threads) {
    const size_t D = sp->D;
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel num_threads(num_threads)
    {
        float *rot = (float *)malloc(sizeof(float) * D);
        float *res = (float *)malloc(sizeof(float) * D);
        uint8_t *idx = (uint8_t *)malloc(D);
#pragma omp for schedule(static)
        for (long long i = 0; i < (long long)n; ++i)
            encode_one(sp, X + (size_t)i * sp->dim, out + (size_t)i * sp->code_size, rot, res, idx);
        free(rot); free(res); free(idx);
    }
}

/* prepareQuery: space_turbo_quant.h:439-460 */
void tqo_prepare_query(const tqo_space *sp, const float *q, float *q_rot, float *s_q,
                       float *norms) {
    const size_t dim = sp->dim, D = sp->D;
    /* In the reference's batch drivers the |q|^2 loop accumulates into a
     * struct member and is compiled as a plain sequential sum (:443-445). */
    float qn2 = 0.0f;
    for (size_t i = 0; i < dim; ++i) {
        float p = q[i] * q[i];
        qn2 = qn2 + p;
    }
    float qn = sqrtf(qn2);
    float qinv = (qn2 > NORMSQ_FLOOR) ? 1.0f / qn : 0.0f;
    for (size_t i = 0; i < D; ++i) q_rot[i] = 0.0f;
    for (size_t i = 0; i < dim; ++i) q_rot[i] = q[i] * qinv;
    rht(q_rot, sp->rot_signs, D, sp->wht_scale);
    memcpy(s_q, q_rot, sizeof(float) * D);
    rht(s_q, sp->qjl_signs, D, sp->wht_scale);
    norms[0] = qn2;
    norms[1] = qn;
}

static inline unsigned code_unit(const uint8_t *packed, size_t i, int bits) {
    if (bits <= 4) {
        uint8_t b = packed[i >> 1];
        return (i & 1) ? (unsigned)(b >> 4) : (unsigned)(b & 0x0F);
    }
    return packed[i];
}

static inline void code_meta(const tqo_space *sp, const uint8_t *code, float m[3]) {
    memcpy(m, code + sp->packed_bytes, 12);
}

/* ---- asymmetric distance as the pinned build computes it --------------------
 * The reference picks distSearchAVX (space_turbo_quant.h:1457-1539) for bits >= 5
 * and distSearchScalarB4 (:951-983) for bits <= 4 on x86 (:280-302).  Under
 * -O3 -ffast-math -march=x86-64-v3 the compiler re-associates both loops; the
 * order below is the one read from the x86 assembly of that build (the
 * assembly of code compiled here from the reference's sources).  Every
 * operation is a single IEEE FP32 rounding (this file is compiled without
 * contraction; fmaf is a fused multiply-add). */

/* A __m256 reduced to a scalar the way both functions end:
 * ((v0 + v4) + (v2 + v6)) + ((v1 + v5) + (v3 + v7)). */
static float hsum8(const float v[8]) {
    float w0 = v[0] + v[4], w1 = v[1] + v[5], w2 = v[2] + v[6], w3 = v[3] + v[7];
    return (w0 + w2) + (w1 + w3);
}

/* A __m128 reduced to a scalar: (u0 + u2) + (u1 + u3). */
static float hsum4(const float u[4]) { return (u[0] + u[2]) + (u[1] + u[3]); }

static inline float signed_s(float s, unsigned bit) { return bit ? s : -s; }

/* distSearchScalarB4 (:951-983), nibble codes.  Byte b holds coordinates 2b
 * (low nibble) and 2b+1 (high nibble).  Per byte the two MSE terms fuse as
 * fma(q[2b], c_lo, q[2b+1] * c_hi) and the two QJL terms add as e_lo + e_hi.
 *  - D >= 64: 32 running sums, byte b into sum b mod 32, in byte order; then
 *    V_j = (A_{16+j} + A_{24+j}) + (A_j + A_{8+j}) and hsum8(V).
 *  - D == 32 (16 bytes left): one 4-lane step whose tree is written out below.
 *  - D <= 16: a sequential loop over bytes.
 * Epilogue: ip = fma(ip_sum, sigma, (scale * gamma) * dot) * |x|, then
 * d = fma(-ip, 2|q|, fma(|x|, |x|, |q|^2)), clamped at 0. */
static float dist_search_b4(const tqo_space *sp, const float *q, const float *s,
                            const float *norms, const uint8_t *code) {
    const size_t D = sp->D, nb = sp->packed_bytes;
    const float *c = sp->centroids;
    float m[3];
    code_meta(sp, code, m);
    /* the reference reads q[2b + 1] of the last byte even at D == 1; it is
     * past the end of its prepared query there, zero here */
    #define QAT(i) ((i) < D ? q[(i)] : 0.0f)
    #define SAT(i) ((i) < D ? s[(i)] : 0.0f)
    float ip = 0.0f, dot = 0.0f;
    size_t b = 0;
    if (D >= 63) {
        float A[32], S[32];
        for (int t = 0; t < 32; ++t) A[t] = S[t] = 0.0f;
        const size_t nb32 = nb & ~(size_t)31;
        for (; b < nb32; b += 32)
            for (int t = 0; t < 32; ++t) {
                const size_t k = b + (size_t)t;
                const unsigned lo = code[k] & 15u, hi = code[k] >> 4;
                const float ph = q[2 * k + 1] * c[hi >> 1];
                A[t] = A[t] + fmaf(q[2 * k], c[lo >> 1], ph);
                S[t] = S[t] + (signed_s(s[2 * k], lo & 1u) + signed_s(s[2 * k + 1], hi & 1u));
            }
        float V[8], W[8];
        for (int j = 0; j < 8; ++j) {
            V[j] = (A[16 + j] + A[24 + j]) + (A[j] + A[8 + j]);
            W[j] = (S[16 + j] + S[24 + j]) + (S[j] + S[8 + j]);
        }
        ip = hsum8(V);
        dot = hsum8(W);
    }
    if (nb - b >= 16) {
        /* bytes b .. b+15 as four groups g of four lanes j: byte b + 4g + j */
        float L[4][4], H[4][4], El[4][4], Eh[4][4];
        for (int g = 0; g < 4; ++g)
            for (int j = 0; j < 4; ++j) {
                const size_t k = b + (size_t)(4 * g + j);
                const unsigned lo = code[k] & 15u, hi = code[k] >> 4;
                L[g][j] = c[lo >> 1];
                H[g][j] = c[hi >> 1];
                El[g][j] = signed_s(SAT(2 * k), lo & 1u);
                Eh[g][j] = signed_s(SAT(2 * k + 1), hi & 1u);
            }
        float U[4], Q4[4];
        for (int j = 0; j < 4; ++j) {
            const size_t k0 = b + (size_t)j, k1 = k0 + 4, k2 = k0 + 8, k3 = k0 + 12;
            const float t1 = fmaf(L[2][j], QAT(2 * k2), QAT(2 * k3) * L[3][j]);
            const float t2 = fmaf(QAT(2 * k0), L[0][j], L[1][j] * QAT(2 * k1));
            const float t3 = fmaf(QAT(2 * k2 + 1), H[2][j], QAT(2 * k3 + 1) * H[3][j]);
            const float t4 = fmaf(QAT(2 * k0 + 1), H[0][j], H[1][j] * QAT(2 * k1 + 1));
            U[j] = ((t4 + t3) + t2) + t1;
            const float p1 = El[0][j] + El[1][j], p2 = El[2][j] + El[3][j];
            const float q1 = Eh[0][j] + Eh[1][j], q3 = Eh[2][j] + Eh[3][j];
            Q4[j] = q3 + (q1 + (p2 + p1));
        }
        ip = ip + hsum4(U);
        dot = dot + hsum4(Q4);
        b += 16;
    }
    for (; b < nb; ++b) {
        const unsigned lo = code[b] & 15u, hi = code[b] >> 4;
        const float ph = c[hi >> 1] * QAT(2 * b + 1);
        ip = ip + fmaf(QAT(2 * b), c[lo >> 1], ph);
        dot = dot + (signed_s(SAT(2 * b + 1), hi & 1u) + signed_s(SAT(2 * b), lo & 1u));
    }
    #undef QAT
    #undef SAT
    float t = (sp->scale * m[1]) * dot;
    t = fmaf(ip, m[2], t) * m[0];
    const float d = fmaf(-t, norms[1] + norms[1], fmaf(m[0], m[0], norms[0]));
    return 0.0f < d ? d : 0.0f;
}

/* distSearchAVX (:1457-1539), byte codes.  D >= 8: eight running sums,
 * coordinate i into sum i mod 8, as fma(c[u >> 1], q[i], sum) and sum + (+-s[i]);
 * ip = hsum8 * sigma, dot = hsum8.  D < 8: a sequential loop of
 * (sigma * q[i]) * c[u >> 1] and +-s[i].  Epilogue:
 * ip = fma(gamma * scale, dot, ip) * |x|, then
 * d = fma(-ip, 2|q|, fma(|x|, |x|, |q|^2)), clamped at 0. */
static float dist_search_b8(const tqo_space *sp, const float *q, const float *s,
                            const float *norms, const uint8_t *code) {
    const size_t D = sp->D;
    const float *c = sp->centroids;
    float m[3];
    code_meta(sp, code, m);
    float ip = 0.0f, dot = 0.0f;
    size_t i = 0;
    if (D >= 8) {
        float A[8], S[8];
        for (int j = 0; j < 8; ++j) A[j] = S[j] = 0.0f;
        for (; i + 8 <= D; i += 8)
            for (int j = 0; j < 8; ++j) {
                const unsigned u = code[i + (size_t)j];
                A[j] = fmaf(c[u >> 1], q[i + (size_t)j], A[j]);
                S[j] = S[j] + signed_s(s[i + (size_t)j], u & 1u);
            }
        ip = hsum8(A) * m[2];
        dot = hsum8(S);
    }
    for (; i < D; ++i) {
        const unsigned u = code[i];
        ip = ip + (m[2] * q[i]) * c[u >> 1];
        dot = dot + signed_s(s[i], u & 1u);
    }
    float t = fmaf(m[1] * sp->scale, dot, ip) * m[0];
    const float d = fmaf(-t, norms[1] + norms[1], fmaf(m[0], m[0], norms[0]));
    return 0.0f < d ? d : 0.0f;
}

static float dist_search(const tqo_space *sp, const float *q_rot, const float *s_q,
                         const float *norms, const uint8_t *code) {
    return sp->bits <= 4 ? dist_search_b4(sp, q_rot, s_q, norms, code)
                         : dist_search_b8(sp, q_rot, s_q, norms, code);
}

/* Symmetric distances in the pinned build's own order (read from the x86
 * assembly of the reference compiled here, and checked bit for bit against it
 * at every padded dim).  Both functions end in the same epilogue:
 *   d = max(0, fma(-(ip + ip), |a| |b|, fma(|a|, |a|, |b| |b|))).
 * The sigma factors leave the per-coordinate products: the loops sum products
 * of centroid values. */
static float sym_epilogue(float ip, float na, float nb) {
    const float d = fmaf(-(ip + ip), na * nb, fmaf(na, na, nb * nb));
    return 0.0f < d ? d : 0.0f;
}

/* distBuildAVX (:1541-1612), byte codes.  D >= 8: eight running sums,
 * coordinate i into sum i mod 8, as fma(c_a[i] * c_b[i], sigma_a sigma_b, sum);
 * ip = hsum8.  D < 8: the same fma in coordinate order into one sum. */
static float dist_build_b8(const tqo_space *sp, const uint8_t *a, const uint8_t *b) {
    const size_t D = sp->D;
    const float *c = sp->centroids;
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    const float sab = ma[2] * mb[2];
    float ip = 0.0f;
    size_t i = 0;
    if (D >= 8) {
        float S[8];
        for (int j = 0; j < 8; ++j) S[j] = 0.0f;
        for (; i + 8 <= D; i += 8)
            for (int j = 0; j < 8; ++j)
                S[j] = fmaf(c[a[i + (size_t)j] >> 1] * c[b[i + (size_t)j] >> 1], sab, S[j]);
        ip = hsum8(S);
    }
    for (; i < D; ++i) ip = fmaf(c[a[i] >> 1] * c[b[i] >> 1], sab, ip);
    return sym_epilogue(ip, ma[0], mb[0]);
}

/* distBuildScalarB4 (:985-1019), nibble codes, as vectorised by the build.
 * Let lo(x, k) / hi(x, k) be the centroid values of byte k's low / high nibble
 * and pair(f, k0, k1) = fma(f(a, k0), f(b, k0), f(a, k1) * f(b, k1)).
 *  - >= 32 bytes, per block of 32 bytes at k and lane j < 8:
 *      s = ((pair(hi, k+16+j, k+24+j) + pair(hi, k+j, k+8+j))
 *           + pair(lo, k+j, k+8+j)) + pair(lo, k+16+j, k+24+j),
 *    S[j] = fma(s * sigma_a, sigma_b, S[j]); ip = hsum8(S).
 *  - 16 bytes (D == 32), lane j < 4: the same with offsets 0/4 and 8/12,
 *    S[j] = (s * sigma_a) * sigma_b; ip = hsum4(S).
 *  - <= 8 bytes: in byte order, ip = fma(fma(lo_a, lo_b, hi_a * hi_b),
 *    sigma_a sigma_b, ip). */
static float dist_build_b4(const tqo_space *sp, const uint8_t *a, const uint8_t *b) {
    const size_t nb = sp->packed_bytes;
    const float *c = sp->centroids;
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    #define LO_(x, k) c[((x)[k] & 15u) >> 1]
    #define HI_(x, k) c[((x)[k] >> 4) >> 1]
    #define PAIR_(F, k0, k1) fmaf(F(a, k0), F(b, k0), F(a, k1) * F(b, k1))
    float ip = 0.0f;
    size_t k = 0;
    if (nb >= 32) {
        float S[8];
        for (int j = 0; j < 8; ++j) S[j] = 0.0f;
        for (; k + 32 <= nb; k += 32)
            for (int j = 0; j < 8; ++j) {
                const size_t l0 = k + (size_t)j, l1 = l0 + 16;
                const float s = ((PAIR_(HI_, l1, l1 + 8) + PAIR_(HI_, l0, l0 + 8)) +
                                 PAIR_(LO_, l0, l0 + 8)) + PAIR_(LO_, l1, l1 + 8);
                S[j] = fmaf(s * ma[2], mb[2], S[j]);
            }
        ip = hsum8(S);
    }
    if (nb - k >= 16) {
        float S4[4];
        for (int j = 0; j < 4; ++j) {
            const size_t l0 = k + (size_t)j, l1 = l0 + 8;
            const float s = ((PAIR_(HI_, l1, l1 + 4) + PAIR_(HI_, l0, l0 + 4)) +
                             PAIR_(LO_, l0, l0 + 4)) + PAIR_(LO_, l1, l1 + 4);
            S4[j] = (s * ma[2]) * mb[2];
        }
        ip = ip + hsum4(S4);
        k += 16;
    }
    const float sab = ma[2] * mb[2];
    for (; k < nb; ++k) ip = fmaf(fmaf(LO_(a, k), LO_(b, k), HI_(a, k) * HI_(b, k)), sab, ip);
    #undef LO_
    #undef HI_
    #undef PAIR_
    return sym_epilogue(ip, ma[0], mb[0]);
}

static float dist_build(const tqo_space *sp, const uint8_t *a, const uint8_t *b) {
    return sp->bits <= 4 ? dist_build_b4(sp, a, b) : dist_build_b8(sp, a, b);
}

void tqo_distance_1_to_n(const tqo_space *sp, const float *q, const uint8_t *codes,
                         size_t n, float *out, int num_threads) {
    float *q_rot = (float *)malloc(sizeof(float) * sp->D);
    float *s_q = (float *)malloc(sizeof(float) * sp->D);
    float norms[2];
    tqo_prepare_query(sp, q, q_rot, s_q, norms);
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel for schedule(static) num_threads(num_threads)
    for (long long i = 0; i < (long long)n; ++i)
        out[i] = dist_search(sp, q_rot, s_q, norms, codes + (size_t)i * sp->code_size);
    free(q_rot); free(s_q);
}

void tqo_distance_m_to_n(const tqo_space *sp, const float *Q, size_t m,
                         const uint8_t *codes, size_t n, float *out, int num_threads) {
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel num_threads(num_threads)
    {
        float *q_rot = (float *)malloc(sizeof(float) * sp->D);
        float *s_q = (float *)malloc(sizeof(float) * sp->D);
        float norms[2];
#pragma omp for schedule(static)
        for (long long qi = 0; qi < (long long)m; ++qi) {
            tqo_prepare_query(sp, Q + (size_t)qi * sp->dim, q_rot, s_q, norms);
            for (size_t i = 0; i < n; ++i)
                out[(size_t)qi * n + i] =
                    dist_search(sp, q_rot, s_q, norms, codes + i * sp->code_size);
        }
        free(q_rot); free(s_q);
    }
}

void tqo_distance_m_to_n_symmetric(const tqo_space *sp, const uint8_t *A, size_t m,
                                   const uint8_t *B, size_t n, float *out,
                                   int num_threads) {
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel for schedule(static) num_threads(num_threads)
    for (long long i = 0; i < (long long)m; ++i)
        for (size_t j = 0; j < n; ++j)
            out[(size_t)i * n + j] =
                dist_build(sp, A + (size_t)i * sp->code_size, B + j * sp->code_size);
}

/* ---- FP64 evaluation of the same formulas --------------------------------- */
static void rht64(double *v, const float *signs, size_t D) {
    for (size_t i = 0; i < D; ++i) v[i] *= (double)signs[i];
    for (size_t step = 1; step < D; step <<= 1)
        for (size_t i = 0; i < D; i += step << 1)
            for (size_t j = 0; j < step; ++j) {
                double a = v[i + j], b = v[i + step + j];
                v[i + j] = a + b;
                v[i + step + j] = a - b;
            }
    double s = 1.0 / sqrt((double)D);
    for (size_t i = 0; i < D; ++i) v[i] *= s;
}

double tqo_distance_f64(const tqo_space *sp, const float *q, const uint8_t *code) {
    const size_t D = sp->D;
    double *q_rot = (double *)calloc(D, sizeof(double));
    double *s_q = (double *)malloc(sizeof(double) * D);
    double qn2 = 0.0;
    for (size_t i = 0; i < sp->dim; ++i) qn2 += (double)q[i] * (double)q[i];
    double qn = sqrt(qn2);
    double qinv = qn > 1e-10 ? 1.0 / qn : 0.0;
    for (size_t i = 0; i < sp->dim; ++i) q_rot[i] = (double)q[i] * qinv;
    rht64(q_rot, sp->rot_signs, D);
    memcpy(s_q, q_rot, sizeof(double) * D);
    rht64(s_q, sp->qjl_signs, D);
    float m[3];
    code_meta(sp, code, m);
    double ip_mse = 0.0, dot = 0.0;
    for (size_t i = 0; i < D; ++i) {
        unsigned u = code_unit(code, i, sp->bits);
        ip_mse += q_rot[i] * (double)sp->centroids[u >> 1];
        dot += s_q[i] * ((u & 1) ? 1.0 : -1.0);
    }
    double xn = m[0], gamma = m[1], sigma = m[2];
    double ip = (ip_mse * sigma + (double)sp->scale * gamma * dot) * xn * qn;
    double d = qn2 + xn * xn - 2.0 * ip;
    free(q_rot); free(s_q);
    return d > 0.0 ? d : 0.0;
}

double tqo_distance_symmetric_f64(const tqo_space *sp, const uint8_t *a, const uint8_t *b) {
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    double ip = 0.0;
    for (size_t i = 0; i < sp->D; ++i)
        ip += ((double)sp->centroids[code_unit(a, i, sp->bits) >> 1] * ma[2]) *
              ((double)sp->centroids[code_unit(b, i, sp->bits) >> 1] * mb[2]);
    ip *= (double)ma[0] * (double)mb[0];
    double d = (double)ma[0] * ma[0] + (double)mb[0] * mb[0] - 2.0 * ip;
    return d > 0.0 ? d : 0.0;
}

/* ---- rotatedCoordsBatch: space_turbo_quant.h:411-435 ----------------------
 * |x|^2 with the same reduction tree as encodeVector (same loop shape), the
 * guard `norm_sq > 1e-20f`, inv_norm = 1 / sqrt(norm_sq), the rotation RHT,
 * var over D, inv_sigma = sqrt(D / var) (guard var > 1e-20f, else 1). */
void tqo_rotated_coords_batch(const tqo_space *sp, const float *X, size_t n, float *out,
                              int num_threads) {
    const size_t dim = sp->dim, D = sp->D;
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel for schedule(static) num_threads(num_threads)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const float *raw = X + (size_t)ii * dim;
        float *dst = out + (size_t)ii * D;
        float norm_sq = tqo_sq_reduce(raw, dim);
        float inv_norm = (norm_sq > 1e-20f) ? 1.0f / sqrtf(norm_sq) : 0.0f;
        for (size_t j = 0; j < D; ++j) dst[j] = 0.0f;
        for (size_t j = 0; j < dim; ++j) dst[j] = raw[j] * inv_norm;
        rht(dst, sp->rot_signs, D, sp->wht_scale);
        float var = tqo_sq_reduce(dst, D);
        float inv_sigma = (var > 1e-20f) ? sqrtf((float)D / var) : 1.0f;
        for (size_t j = 0; j < D; ++j) dst[j] = dst[j] * inv_sigma;
    }
}

/* ---- QJL-corrected symmetric distances: space_turbo_quant.h:483-572, 731-945
 * Sums are evaluated in index order as written in the reference's scalar
 * functions (its build may vectorise them; the bar for distances is 1e-5). */
static float pi_over_2d(const tqo_space *sp) {
    return (float)M_PI / (2.0f * (float)sp->D);
}

static float clampf_(float v, float lim) {
    return v > lim ? lim : (v < -lim ? -lim : v);
}

/* distBuildFullScalar (:731-800) */
static float dist_build_full(const tqo_space *sp, const uint8_t *a, const uint8_t *b,
                             float *ra, float *rb) {
    const size_t D = sp->D;
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    float ip_mse = 0.0f;
    for (size_t i = 0; i < D; ++i) {
        float ca = sp->centroids[code_unit(a, i, sp->bits) >> 1] * ma[2];
        float cb = sp->centroids[code_unit(b, i, sp->bits) >> 1] * mb[2];
        ip_mse = ip_mse + ca * cb;
        ra[i] = ca;
        rb[i] = cb;
    }
    rht(ra, sp->qjl_signs, D, sp->wht_scale);
    rht(rb, sp->qjl_signs, D, sp->wht_scale);
    float t_ab = 0.0f, t_ba = 0.0f, t_ss = 0.0f;
    for (size_t i = 0; i < D; ++i) {
        float sa = (code_unit(a, i, sp->bits) & 1) ? 1.0f : -1.0f;
        float sb = (code_unit(b, i, sp->bits) & 1) ? 1.0f : -1.0f;
        t_ab = t_ab + ra[i] * sb;
        t_ba = t_ba + sa * rb[i];
        t_ss = t_ss + sa * sb;
    }
    float term2 = sp->scale * mb[1] * t_ab;
    float term3 = sp->scale * ma[1] * t_ba;
    float term4 = pi_over_2d(sp) * ma[1] * mb[1] * t_ss;
    float corr = clampf_(term2 + term3 + term4, fabsf(ip_mse));
    float ip = (ip_mse + corr) * ma[0] * mb[0];
    float d = ma[0] * ma[0] + mb[0] * mb[0] - 2.0f * ip;
    return d > 0.0f ? d : 0.0f;
}

/* distBuildLightScalar (:902-945) */
static float dist_build_light(const tqo_space *sp, const uint8_t *a, const uint8_t *b) {
    const size_t D = sp->D;
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    float ip_mse = 0.0f;
    int agree = 0;
    for (size_t i = 0; i < D; ++i) {
        unsigned ua = code_unit(a, i, sp->bits), ub = code_unit(b, i, sp->bits);
        ip_mse = ip_mse + (sp->centroids[ua >> 1] * ma[2]) * (sp->centroids[ub >> 1] * mb[2]);
        agree += ((ua ^ ub) & 1u) == 0 ? 1 : 0;
    }
    float dot_signs = (float)(2 * agree - (int)D);
    float corr = clampf_(pi_over_2d(sp) * ma[1] * mb[1] * dot_signs, fabsf(ip_mse));
    float ip = (ip_mse + corr) * ma[0] * mb[0];
    float d = ma[0] * ma[0] + mb[0] * mb[0] - 2.0f * ip;
    return d > 0.0f ? d : 0.0f;
}

/* prepareSymmetricQuery (:499-535): recon_q = RHT_qjl(c[idx] * sigma),
 * sign_q = +-1, s[0..4] = norm, gamma, sigma, scale * gamma,
 * (pi / (2 D)) * gamma. */
void tqo_prepare_symmetric(const tqo_space *sp, const uint8_t *code, float *recon_q,
                           float *sign_q, float *s) {
    const size_t D = sp->D;
    float m[3];
    code_meta(sp, code, m);
    for (size_t i = 0; i < D; ++i) {
        unsigned u = code_unit(code, i, sp->bits);
        recon_q[i] = sp->centroids[u >> 1] * m[2];
        sign_q[i] = (u & 1) ? 1.0f : -1.0f;
    }
    rht(recon_q, sp->qjl_signs, D, sp->wht_scale);
    s[0] = m[0];
    s[1] = m[1];
    s[2] = m[2];
    s[3] = sp->scale * m[1];
    s[4] = pi_over_2d(sp) * m[1];
}

/* distBuildFullPreparedScalar (:808-878) */
static float dist_build_full_prepared(const tqo_space *sp, const float *recon_q,
                                      const float *sign_q, const float *s, const uint8_t *b,
                                      float *rb) {
    const size_t D = sp->D;
    float mb[3];
    code_meta(sp, b, mb);
    for (size_t i = 0; i < D; ++i)
        rb[i] = sp->centroids[code_unit(b, i, sp->bits) >> 1] * mb[2];
    rht(rb, sp->qjl_signs, D, sp->wht_scale);
    float d_rr = 0.0f, d_rs = 0.0f, d_sr = 0.0f, d_ss = 0.0f;
    for (size_t i = 0; i < D; ++i) {
        float sb = (code_unit(b, i, sp->bits) & 1) ? 1.0f : -1.0f;
        d_rr = d_rr + recon_q[i] * rb[i];
        d_rs = d_rs + recon_q[i] * sb;
        d_sr = d_sr + sign_q[i] * rb[i];
        d_ss = d_ss + sign_q[i] * sb;
    }
    float term2 = sp->scale * mb[1] * d_rs;
    float term3 = s[3] * d_sr;
    float term4 = s[4] * mb[1] * d_ss;
    float corr = clampf_(term2 + term3 + term4, fabsf(d_rr));
    float ip = (d_rr + corr) * s[0] * mb[0];
    float d = s[0] * s[0] + mb[0] * mb[0] - 2.0f * ip;
    return d > 0.0f ? d : 0.0f;
}

void tqo_distance_m_to_n_symmetric_qjl(const tqo_space *sp, const uint8_t *A, size_t m,
                                       const uint8_t *B, size_t n, float *out, int variant,
                                       int num_threads) {
    const size_t D = sp->D, cs = sp->code_size;
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel num_threads(num_threads)
    {
        float *ra = (float *)malloc(sizeof(float) * D);
        float *rb = (float *)malloc(sizeof(float) * D);
        float *sq = (float *)malloc(sizeof(float) * D);
        float s[5];
#pragma omp for schedule(static)
        for (long long i = 0; i < (long long)m; ++i) {
            const uint8_t *a = A + (size_t)i * cs;
            if (variant == TQO_SYM_FULL_PREPARED) tqo_prepare_symmetric(sp, a, ra, sq, s);
            for (size_t j = 0; j < n; ++j) {
                const uint8_t *b = B + j * cs;
                float d;
                if (variant == TQO_SYM_LIGHT) d = dist_build_light(sp, a, b);
                else if (variant == TQO_SYM_FULL) d = dist_build_full(sp, a, b, ra, rb);
                else d = dist_build_full_prepared(sp, ra, sq, s, b, rb);
                out[(size_t)i * n + j] = d;
            }
        }
        free(ra); free(rb); free(sq);
    }
}

void tqo_distance_1_to_n_symmetric_full(const tqo_space *sp, const float *recon_q,
                                        const float *sign_q, const float *s,
                                        const uint8_t *B, size_t n, float *out,
                                        int num_threads) {
    const size_t D = sp->D;
    if (num_threads <= 0) num_threads = 1;
#pragma omp parallel num_threads(num_threads)
    {
        float *rb = (float *)malloc(sizeof(float) * D);
#pragma omp for schedule(static)
        for (long long j = 0; j < (long long)n; ++j)
            out[j] = dist_build_full_prepared(sp, recon_q, sign_q, s,
                                              B + (size_t)j * sp->code_size, rb);
        free(rb);
    }
}

/* FP64 evaluation of the three corrected formulas on the same codes (the
 * prepared variant's ip_mse is the post-Hadamard dot, equal in exact
 * arithmetic to the full variant's pre-Hadamard one). */
double tqo_distance_symmetric_qjl_f64(const tqo_space *sp, const uint8_t *a, const uint8_t *b,
                                      int variant) {
    const size_t D = sp->D;
    float ma[3], mb[3];
    code_meta(sp, a, ma);
    code_meta(sp, b, mb);
    double *ra = (double *)malloc(sizeof(double) * D);
    double *rb = (double *)malloc(sizeof(double) * D);
    double ip_mse = 0.0, t_ab = 0.0, t_ba = 0.0, t_ss = 0.0;
    for (size_t i = 0; i < D; ++i) {
        ra[i] = (double)sp->centroids[code_unit(a, i, sp->bits) >> 1] * ma[2];
        rb[i] = (double)sp->centroids[code_unit(b, i, sp->bits) >> 1] * mb[2];
        ip_mse += ra[i] * rb[i];
    }
    rht64(ra, sp->qjl_signs, D);
    rht64(rb, sp->qjl_signs, D);
    for (size_t i = 0; i < D; ++i) {
        double sa = (code_unit(a, i, sp->bits) & 1) ? 1.0 : -1.0;
        double sb = (code_unit(b, i, sp->bits) & 1) ? 1.0 : -1.0;
        t_ab += ra[i] * sb;
        t_ba += sa * rb[i];
        t_ss += sa * sb;
    }
    free(ra); free(rb);
    const double p2d = M_PI / (2.0 * (double)D), scale = sqrt(M_PI / 2.0) / sqrt((double)D);
    double corr = p2d * ma[1] * mb[1] * t_ss;
    if (variant != TQO_SYM_LIGHT) corr += scale * mb[1] * t_ab + scale * ma[1] * t_ba;
    double lim = fabs(ip_mse);
    corr = corr > lim ? lim : (corr < -lim ? -lim : corr);
    double ip = (ip_mse + corr) * ma[0] * mb[0];
    double d = (double)ma[0] * ma[0] + (double)mb[0] * mb[0] - 2.0 * ip;
    return d > 0.0 ? d : 0.0;
}
