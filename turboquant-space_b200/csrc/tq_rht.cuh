// tq_rht.cuh -- device helpers shared by the sm_100a kernels that rotate,
// reduce or quantize vectors (tq_kernels.cu, tq_symq.cu): the swizzled
// shared-memory FWHT, the reference's sum-of-squares tree, the quantizer and
// the shared table block.  Header-only; every helper is an inline device
// function in an unnamed namespace.
#pragma once

#include <cstdint>

#include "tq_internal.h"

namespace tq {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float f32_bits(uint32_t u) { return __uint_as_float(u); }

// Bijective index swizzle of a vector held in shared memory: the low 5 bits
// (the bank) are XORed with bits 5-9 and 10-14.  It makes the FWHT passes'
// group loads (contiguous or strided) and the 8-lane reduction chains
// bank-conflict-free for the power-of-two sizes used here.
__device__ __forceinline__ int swz(int e) { return e ^ (((e >> 5) ^ (e >> 10)) & 31); }

// Multiply by the +-1 sign of element e (bit set = +1): an exact sign flip.
__device__ __forceinline__ float apply_sign(float x, const uint32_t *mask, int e) {
    const uint32_t bit = (mask[e >> 5] >> (e & 31)) & 1u;
    return __uint_as_float(__float_as_uint(x) ^ ((bit ^ 1u) << 31));
}

// ---------------------------------------------------------------------------
// Warp-level FWHT on a swizzled shared-memory vector of D = 2^LOG_D floats.
// The butterflies run in stage order stride 1, 2, 4, ..., D/2 exactly as
// whtInplaceScalar (turbo_quant.h:46-60) -- each output is a single rounding
// of a + b or a - b of the previous stage, so the result is bit-identical.
// Stages are grouped into passes of up to 5 (2^5 values per group held in
// registers); a pass reads and writes the vector once.
//   pass 1 also applies the pre-multiply (x * pre, rounded) and the sign flip
//   (randomizedHadamard, turbo_quant.h:95-97); the last pass applies the
//   1/sqrt(D) normalisation (turbo_quant.h:69-71).
// ---------------------------------------------------------------------------
template <int LOG_D>
struct FwhtPlan {
    static constexpr int PL = (LOG_D - 5 < 1) ? 1 : ((LOG_D - 5 > 5) ? 5 : LOG_D - 5);
};

template <int LOG_D, int S0, int R, bool FIRST, bool LAST, bool PREMUL>
__device__ __forceinline__ void fwht_pass(float *buf, int lane, float pre, const uint32_t *mask,
                                          float post) {
    constexpr int D = 1 << LOG_D;
    constexpr int NR = 1 << R;
    constexpr int NG = D / NR;
    constexpr int G = (NG + 31) / 32;
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int o = lane + 32 * gi;
        if ((NG & 31) != 0 && o >= NG) break;
        const int base = (o & ((1 << S0) - 1)) | ((o >> S0) << (S0 + R));
        float v[NR];
#pragma unroll
        for (int t = 0; t < NR; ++t) {
            const int e = base | (t << S0);
            float x = buf[swz(e)];
            if constexpr (FIRST) {
                if constexpr (PREMUL) x = __fmul_rn(x, pre);
                x = apply_sign(x, mask, e);
            }
            v[t] = x;
        }
#pragma unroll
        for (int s = 0; s < R; ++s) {
#pragma unroll
            for (int t = 0; t < NR; ++t) {
                if (!(t & (1 << s))) {
                    const float a = v[t], b = v[t | (1 << s)];
                    v[t] = __fadd_rn(a, b);
                    v[t | (1 << s)] = __fsub_rn(a, b);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < NR; ++t) {
            float x = v[t];
            if constexpr (LAST) x = __fmul_rn(x, post);
            buf[swz(base | (t << S0))] = x;
        }
    }
}

template <int LOG_D, int S0, bool PREMUL>
__device__ __forceinline__ void fwht_from(float *buf, int lane, float pre, const uint32_t *mask,
                                          float post) {
    if constexpr (S0 < LOG_D) {
        constexpr int PL = FwhtPlan<LOG_D>::PL;
        constexpr int R = (LOG_D - S0 < PL) ? (LOG_D - S0) : PL;
        fwht_pass<LOG_D, S0, R, S0 == 0, S0 + R == LOG_D, PREMUL>(buf, lane, pre, mask, post);
        __syncwarp();
        fwht_from<LOG_D, S0 + R, PREMUL>(buf, lane, pre, mask, post);
    }
}

// ---------------------------------------------------------------------------
// The reference's FP32 sum of squares as its pinned build evaluates it
// (space_turbo_quant.h:343-344, 354-355, 370-371; restated in the CPU
// checker): 8 accumulators acc[k] += x[i]^2 for i = k (mod 8) with separate
// multiply and add roundings; t[k] = acc[k] + acc[k+4]; s = (t0+t2)+(t1+t3);
// a 4-wide FMA step over the next 4 leftovers (from t, or from zero when
// n < 8) and a scalar FMA tail.  Evaluated by the 8 lanes of group
// g = lane/8 on the swizzled vector `buf`; all 8 lanes return the sum.  All
// 32 lanes must call it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float chain_sq_reduce(const float *buf, int n, int lane) {
    const int k = lane & 7;
    const int n8 = n & ~7;
    float acc = 0.0f;
#pragma unroll 8
    for (int i = k; i < n8; i += 8) {
        const float x = buf[swz(i)];
        acc = __fadd_rn(acc, __fmul_rn(x, x));
    }
    const float hi = __shfl_down_sync(kFull, acc, 4, 8);
    const float t = __fadd_rn(acc, hi);
    float t0 = __shfl_sync(kFull, t, 0, 8);
    float t1 = __shfl_sync(kFull, t, 1, 8);
    float t2 = __shfl_sync(kFull, t, 2, 8);
    float t3 = __shfl_sync(kFull, t, 3, 8);
    float s = __fadd_rn(__fadd_rn(t0, t2), __fadd_rn(t1, t3));
    int b = n8, r = n - n8;
    if (r >= 4) {
        const float x0 = buf[swz(b)], x1 = buf[swz(b + 1)];
        const float x2 = buf[swz(b + 2)], x3 = buf[swz(b + 3)];
        t0 = __fmaf_rn(x0, x0, t0);
        t1 = __fmaf_rn(x1, x1, t1);
        t2 = __fmaf_rn(x2, x2, t2);
        t3 = __fmaf_rn(x3, x3, t3);
        s = __fadd_rn(__fadd_rn(t0, t2), __fadd_rn(t1, t3));
        b += 4;
        r -= 4;
    }
    for (int j = 0; j < r; ++j) {
        const float x = buf[swz(b + j)];
        s = __fmaf_rn(x, x, s);
    }
    return s;
}

// quantize (space_turbo_quant.h:332-337): idx = #{j : z > B[j]}.
// nb <= 15: the direct count.  Otherwise bucket j = clamp(fma(z, S, C)) of a
// 2048-entry table gives lo = the number of boundaries every z of that bucket
// exceeds, and only the next qlut_k boundaries are compared.  The host builds
// the table from the exact float range of each bucket, so the count is exact.
__device__ __forceinline__ int quantize(float z, const Params &P, const float *bnd,
                                        const uint8_t *qlut) {
    int idx = 0;
    if (P.lutq) {
        float y = __fmaf_rn(z, P.qlut_s, P.qlut_c);
        y = fminf(fmaxf(y, 0.0f), (float)(kQlutBuckets - 1));
        idx = qlut[(int)y];
        const int lo = idx;
        for (int t = 0; t < P.qlut_k; ++t) idx += (z > bnd[lo + t]) ? 1 : 0;
    } else {
        for (int t = 0; t < P.nb; ++t) idx += (z > bnd[t]) ? 1 : 0;
    }
    return idx & 0xFF;  // the reference accumulates into a uint8_t
}

// quantize with one shared loop: the bucket table narrows the range to
// [lo, lo + k) (k = 1 for every Lloyd-Max table of b = 2..9), the direct count
// (no table) to [0, nb).  Kept out of line of the unrolled callers: one loop.
__device__ __forceinline__ int quantize_compact(float z, const Params &P, const float *bnd,
                                                const uint8_t *qlut) {
    int idx = 0, t1 = P.nb;
    if (P.lutq) {
        float y = __fmaf_rn(z, P.qlut_s, P.qlut_c);
        y = fminf(fmaxf(y, 0.0f), (float)(kQlutBuckets - 1));
        idx = qlut[(int)y];
        if (P.qlut_k == 1) return (idx + ((z > bnd[idx]) ? 1 : 0)) & 0xFF;
        t1 = idx + P.qlut_k;
    }
    const int t0 = idx;
#pragma unroll 1
    for (int t = t0; t < t1; ++t) idx += (z > bnd[t]) ? 1 : 0;
    return idx & 0xFF;
}

// Shared table block of the encode / prepare kernels.
constexpr int kTabCentOff = 0;                                  // float[256]
constexpr int kTabBndOff = kTabCentOff + 4 * kMaxLevels;        // float[256 + 8]
constexpr int kTabRotOff = kTabBndOff + 4 * (kMaxLevels + 8);   // u32[256]
constexpr int kTabQjlOff = kTabRotOff + 4 * 256;                // u32[256]
constexpr int kTabQlutOff = kTabQjlOff + 4 * 256;               // u8[2048]
constexpr int kTabBytes = kTabQlutOff + kQlutBuckets;           // 6176 (16-aligned)
static_assert(kTabBytes % 16 == 0, "table block must keep 16-byte alignment");

// flagged: the bucket table with bit 7 set on the buckets that hold a
// boundary (T.qlutf, for P.qflag) instead of the plain one.
__device__ __forceinline__ void load_tables(unsigned char *smem, const Params &P,
                                            const DevTables &T, bool quant, bool flagged = false) {
    float *cent = reinterpret_cast<float *>(smem + kTabCentOff);
    float *bnd = reinterpret_cast<float *>(smem + kTabBndOff);
    uint32_t *rot = reinterpret_cast<uint32_t *>(smem + kTabRotOff);
    uint32_t *qjl = reinterpret_cast<uint32_t *>(smem + kTabQjlOff);
    uint8_t *qlut = smem + kTabQlutOff;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int mw = (P.D + 31) >> 5;
    for (int i = tid; i < mw; i += nt) {
        rot[i] = T.rot_mask[i];
        qjl[i] = T.qjl_mask[i];
    }
    if (quant) {
        for (int i = tid; i < P.levels; i += nt) cent[i] = T.centroids[i];
        for (int i = tid; i < P.nb + kQlutMaxK; i += nt) bnd[i] = T.boundaries[i];
        if (P.lutq) {
            const uint8_t *src = flagged ? T.qlutf : T.qlut;
            for (int i = tid; i < kQlutBuckets; i += nt) qlut[i] = src[i];
        }
    }
}

__host__ __device__ __forceinline__ int align16(int x) { return (x + 15) & ~15; }

}  // namespace
}  // namespace tq
