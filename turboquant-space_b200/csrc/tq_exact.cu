// tq_exact.cu -- the reference's asymmetric distance replayed on the GPU in the
// summation order of the reference's own Release build, and the serving
// path's exact top-k stages built on it.
//
// The reference evaluates distSearchScalarB4 (space_turbo_quant.h:951-983) for
// bits <= 4 and distSearchAVX (:1457-1539) for bits >= 5 on x86 (:280-302).
// Compiled with its Release flags (-O3 -ffast-math -march=x86-64-v3), both
// loops are re-associated by the compiler; the orders below are the ones that
// build executes (read from its x86 assembly, and pinned bit for bit against
// it on every padded dim by the CPU checker's tests):
//
//   nibble codes, byte b = coordinates 2b (low nibble) and 2b+1 (high):
//     pair_b = fma(q[2b], c[lo >> 1], q[2b+1] * c[hi >> 1]),
//     sign_b = (+-s[2b]) + (+-s[2b+1]);
//     D >= 64: 32 running sums, byte b into sum b mod 32 in byte order, then
//              V_j = (A_{16+j} + A_{24+j}) + (A_j + A_{8+j}), hsum8(V);
//     D == 32: one 16-byte step with the tree written out in exact_b4;
//     D <= 16: a sequential loop;
//     ip = fma(sum, sigma, (scale * gamma) * dot) * |x|.
//   byte codes: D >= 8: 8 running sums, coordinate i into sum i mod 8 as
//     fma(c[u >> 1], q[i], sum); ip = hsum8 * sigma, dot = hsum8;
//     D < 8: a sequential loop of (sigma * q[i]) * c[u >> 1];
//     ip = fma(gamma * scale, dot, ip) * |x|.
//   both: d = max(0, fma(-ip, 2|q|, fma(|x|, |x|, |q|^2))),
//   hsum8(v) = ((v0 + v4) + (v2 + v6)) + ((v1 + v5) + (v3 + v7)).
//
// Every operation below is one IEEE FP32 rounding (explicit _rn intrinsics:
// nvcc would otherwise contract a multiply and an add into an FMA).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>

#include "tq_exact.h"
#include "tq_mton.h"

namespace tq {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNoIdx = INT_MAX;

// Error bound of the distance epilogues, against |q|^2 + max |x|^2 (the
// tensor pass's own bound, kappa, comes with each launch; derivation in
// rescore_kernel).
constexpr float kKappaEpi = 1e-6f;
constexpr float kDegenerateG = 1e-20f;

__device__ __forceinline__ float sgn_s(float s, unsigned bit) { return bit ? s : -s; }

// A 32-bit word of a code in global or shared memory (generic load).
__device__ __forceinline__ uint32_t ld_u32(const uint8_t *p, bool al4) {
    if (al4) return *reinterpret_cast<const unsigned int *>(p);
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

__device__ __forceinline__ float ld_f32(const uint8_t *p, bool al4) { return __uint_as_float(ld_u32(p, al4)); }

__device__ __forceinline__ float hsum8(const float (&v)[8]) {
    const float w0 = __fadd_rn(v[0], v[4]), w1 = __fadd_rn(v[1], v[5]);
    const float w2 = __fadd_rn(v[2], v[6]), w3 = __fadd_rn(v[3], v[7]);
    return __fadd_rn(__fadd_rn(w0, w2), __fadd_rn(w1, w3));
}

__device__ __forceinline__ float hsum4(const float (&u)[4]) {
    return __fadd_rn(__fadd_rn(u[0], u[2]), __fadd_rn(u[1], u[3]));
}

__device__ __forceinline__ float finish_dist(float t, float xn, float qn2, float qn) {
    const float d = __fmaf_rn(-t, __fadd_rn(qn, qn), __fmaf_rn(xn, xn, qn2));
    return 0.0f < d ? d : 0.0f;
}

// distSearchScalarB4 in the reference build's order (nibble codes, pb = D/2).
__device__ float exact_b4(const float *__restrict__ c, const float *__restrict__ q,
                          const float *__restrict__ s, float qn2, float qn, float scale, int D,
                          int nb, const uint8_t *__restrict__ code, bool al4) {
    float ip = 0.0f, dot = 0.0f;
    int b = 0;
    if (D >= 63) {
        float A[32], S[32];
#pragma unroll
        for (int t = 0; t < 32; ++t) A[t] = S[t] = 0.0f;
        const int nb32 = nb & ~31;
#pragma unroll 1
        for (; b < nb32; b += 32) {
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                const uint32_t x = ld_u32(code + b + 4 * w, al4);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int t = 4 * w + e, k = b + t;
                    const unsigned lo = (x >> (8 * e)) & 15u, hi = (x >> (8 * e + 4)) & 15u;
                    const float2 qq = __ldg(reinterpret_cast<const float2 *>(q) + k);
                    const float2 ss = __ldg(reinterpret_cast<const float2 *>(s) + k);
                    const float ph = __fmul_rn(qq.y, c[hi >> 1]);
                    A[t] = __fadd_rn(A[t], __fmaf_rn(qq.x, c[lo >> 1], ph));
                    S[t] = __fadd_rn(S[t], __fadd_rn(sgn_s(ss.x, lo & 1u), sgn_s(ss.y, hi & 1u)));
                }
            }
        }
        float V[8], W[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            V[j] = __fadd_rn(__fadd_rn(A[16 + j], A[24 + j]), __fadd_rn(A[j], A[8 + j]));
            W[j] = __fadd_rn(__fadd_rn(S[16 + j], S[24 + j]), __fadd_rn(S[j], S[8 + j]));
        }
        ip = hsum8(V);
        dot = hsum8(W);
    }
    if (nb - b >= 16) {
        // bytes b .. b+15 as four groups g of four lanes j: byte b + 4g + j
        float L[16], H[16], El[16], Eh[16], Qe[16], Qo[16];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint32_t x = ld_u32(code + b + 4 * w, al4);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int t = 4 * w + e, k = b + t;
                const unsigned lo = (x >> (8 * e)) & 15u, hi = (x >> (8 * e + 4)) & 15u;
                const float2 qq = __ldg(reinterpret_cast<const float2 *>(q) + k);
                const float2 ss = __ldg(reinterpret_cast<const float2 *>(s) + k);
                L[t] = c[lo >> 1];
                H[t] = c[hi >> 1];
                El[t] = sgn_s(ss.x, lo & 1u);
                Eh[t] = sgn_s(ss.y, hi & 1u);
                Qe[t] = qq.x;
                Qo[t] = qq.y;
            }
        }
        float U[4], Q4[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k0 = j, k1 = 4 + j, k2 = 8 + j, k3 = 12 + j;
            const float t1 = __fmaf_rn(L[k2], Qe[k2], __fmul_rn(Qe[k3], L[k3]));
            const float t2 = __fmaf_rn(Qe[k0], L[k0], __fmul_rn(L[k1], Qe[k1]));
            const float t3 = __fmaf_rn(Qo[k2], H[k2], __fmul_rn(Qo[k3], H[k3]));
            const float t4 = __fmaf_rn(Qo[k0], H[k0], __fmul_rn(H[k1], Qo[k1]));
            U[j] = __fadd_rn(__fadd_rn(__fadd_rn(t4, t3), t2), t1);
            const float p1 = __fadd_rn(El[k0], El[k1]), p2 = __fadd_rn(El[k2], El[k3]);
            const float q1 = __fadd_rn(Eh[k0], Eh[k1]), q3 = __fadd_rn(Eh[k2], Eh[k3]);
            Q4[j] = __fadd_rn(q3, __fadd_rn(q1, __fadd_rn(p2, p1)));
        }
        ip = __fadd_rn(ip, hsum4(U));
        dot = __fadd_rn(dot, hsum4(Q4));
        b += 16;
    }
#pragma unroll 1
    for (; b < nb; ++b) {
        const unsigned byte = code[b], lo = byte & 15u, hi = byte >> 4;
        const float ph = __fmul_rn(c[hi >> 1], q[2 * b + 1]);
        ip = __fadd_rn(ip, __fmaf_rn(q[2 * b], c[lo >> 1], ph));
        dot = __fadd_rn(dot, __fadd_rn(sgn_s(s[2 * b + 1], hi & 1u), sgn_s(s[2 * b], lo & 1u)));
    }
    const float xn = ld_f32(code + nb, al4), g = ld_f32(code + nb + 4, al4);
    const float sig = ld_f32(code + nb + 8, al4);
    float t = __fmul_rn(__fmul_rn(scale, g), dot);
    t = __fmul_rn(__fmaf_rn(ip, sig, t), xn);
    return finish_dist(t, xn, qn2, qn);
}

// distSearchAVX in the reference build's order (byte codes, pb = D).
__device__ float exact_b8(const float *__restrict__ c, const float *__restrict__ q,
                          const float *__restrict__ s, float qn2, float qn, float scale, int D,
                          const uint8_t *__restrict__ code, bool al4) {
    const float xn = ld_f32(code + D, al4), g = ld_f32(code + D + 4, al4);
    const float sig = ld_f32(code + D + 8, al4);
    float ip = 0.0f, dot = 0.0f;
    int i = 0;
    if (D >= 8) {
        float A[8], S[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) A[j] = S[j] = 0.0f;
#pragma unroll 1
        for (; i + 8 <= D; i += 8) {
            const uint32_t x0 = ld_u32(code + i, al4), x1 = ld_u32(code + i + 4, al4);
            const float4 q0 = __ldg(reinterpret_cast<const float4 *>(q + i));
            const float4 q1 = __ldg(reinterpret_cast<const float4 *>(q + i) + 1);
            const float4 s0 = __ldg(reinterpret_cast<const float4 *>(s + i));
            const float4 s1 = __ldg(reinterpret_cast<const float4 *>(s + i) + 1);
            const float qv[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            const float sv[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const unsigned u = ((j < 4 ? x0 : x1) >> (8 * (j & 3))) & 255u;
                A[j] = __fmaf_rn(c[u >> 1], qv[j], A[j]);
                S[j] = __fadd_rn(S[j], sgn_s(sv[j], u & 1u));
            }
        }
        ip = __fmul_rn(hsum8(A), sig);
        dot = hsum8(S);
    }
#pragma unroll 1
    for (; i < D; ++i) {
        const unsigned u = code[i];
        ip = __fadd_rn(ip, __fmul_rn(__fmul_rn(sig, q[i]), c[u >> 1]));
        dot = __fadd_rn(dot, sgn_s(s[i], u & 1u));
    }
    const float t = __fmul_rn(__fmaf_rn(__fmul_rn(g, scale), dot, ip), xn);
    return finish_dist(t, xn, qn2, qn);
}

template <bool NIBBLE>
__device__ __forceinline__ float exact_dist(const Params &P, const float *c, const float *q,
                                            const float *s, float qn2, float qn, const uint8_t *code,
                                            bool al4) {
    if (NIBBLE) return exact_b4(c, q, s, qn2, qn, P.scale, P.D, P.pb, code, al4);
    return exact_b8(c, q, s, qn2, qn, P.scale, P.D, code, al4);
}

__device__ __forceinline__ bool better(float d, int i, float bd, int bi) {
    return d < bd || (d == bd && i < bi);
}

// Sorted insert of (d, i) into the ascending list of k entries; returns the
// new k-th entry through kd / ki.  Out of line: few candidates pass a
// thread's threshold.
__device__ __noinline__ void list_insert(float *bd, int *bi, int k, float d, int i, float *kd,
                                         int *ki) {
    float cd = d;
    int cx = i;
#pragma unroll 1
    for (int u = 0; u < k; ++u) {
        if (better(cd, cx, bd[u], bi[u])) {
            const float od = bd[u];
            const int ox = bi[u];
            bd[u] = cd;
            bi[u] = cx;
            cd = od;
            cx = ox;
        }
    }
    *kd = bd[k - 1];
    *ki = bi[k - 1];
}

// k rounds of a warp arg-min over the lanes' ascending lists (each of k
// entries): lane u receives the u-th smallest (distance, index) of the warp;
// lanes u >= k receive (+inf, no index).
__device__ void warp_merge(const float *bd, const int *bi, int k, int lane, float &my_d, int &my_i) {
    int head = 0;
    my_d = INFINITY;
    my_i = kNoIdx;
#pragma unroll 1
    for (int u = 0; u < k; ++u) {
        const float hd = head < k ? bd[head] : INFINITY;
        const int hx = head < k ? bi[head] : kNoIdx;
        float wd = hd;
        int wx = hx;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float od = __shfl_xor_sync(kFull, wd, off);
            const int ox = __shfl_xor_sync(kFull, wx, off);
            if (better(od, ox, wd, wx)) {
                wd = od;
                wx = ox;
            }
        }
        if (hx == wx && hd == wd && wx != kNoIdx) ++head;  // the winning lane pops its head
        if (lane == u) {
            my_d = wd;
            my_i = wx;
        }
    }
}

// The centroid table in shared memory, zero past the space's levels (an
// index no encoder writes reads 0 in every kernel of this file alike).
__device__ __forceinline__ void load_centroids(float *sc, const float *centroids, int levels) {
    for (int i = threadIdx.x; i < kMaxLevels; i += blockDim.x) sc[i] = i < levels ? centroids[i] : 0.0f;
    __syncthreads();
}

struct RescoreArgs {
    Params P;
    const float *centroids;
    float cmax;
    const int *m_dev;
    int kc, k;
    const float *cand_d;
    const long long *cand_i;
    const float *q_rot, *s_q, *norms;
    const uint8_t *codes;
    size_t n;
    bool al4;
    const float *bound;
    float kappa, kappa_t, bound_scale;
    float *out_d;
    long long *out_i;
    int *fail_rows;
    float *thr, *tthr;
    int *counters;
};

// One warp per query row, lane l on candidate l.
//
// The certificate.  Let d'_j be the tensor pass's distance of code j and d_j
// the reference's.  If |d'_j - d_j| <= eps for every j, a code outside the kc
// candidates has d_j >= d'_j - eps >= d'_(kc) - eps (the candidates are the kc
// smallest d'), so when the k-th exact distance among the candidates is below
// d'_(kc) - eps no excluded code can enter the top-k, ties included.
//
// eps.  The tensor pass forms ip = sum_i a_i b_i from hi + lo BF16 pairs:
// a_i = q_rot_i, b_i = sigma c_i / g (the centroid half; g = scale gamma) and
// a_i = s_q_i, b_i = +-1 (the sign half), scaled by g |x| |q|.  Per term, the
// dropped lo*lo product and the pairs' residuals are below 3 * 2^-16 |a_i b_i|;
// each 16-deep MMA step is assumed to add at most 2^-20 (|acc| + sum |p|), and
// a chunk of at most 8 K blocks issues at most 96 MMAs into one accumulator
// from zero (96 * 2^-20 of the chunk's |terms|); promotions, the planes' FP32
// roundings and the reference's own FP32 sums (chains of at most D/64 + 8
// adds) add a few 1e-7.  Their sum, 1.4e-4, is taken as kappa = 2.5e-4 of
// sum_i |terms| (a pass with more MMAs per accumulator, as the whole-K
// variant, brings a kappa grown with their count: tc_topk_kappa), and
//   sum_i |terms| <= |q| (cmax sigma_j |x_j| sum|q_rot| + scale gamma_j |x_j| sum|s_q|),
// bounded with the index-wide maxima of sigma |x| and scale gamma |x|.  The
// distance epilogues of both sides add kKappaEpi (|q|^2 + max |x|^2), and a
// code with g < 1e-20 (whose sign half the tensor pass drops) at most
// 2 |q| sum|s_q| 1e-20 max|x|.  Each candidate is checked against the same
// eps; a candidate outside it is counted and fails its row.
template <bool NIBBLE>
__global__ void __launch_bounds__(256) rescore_kernel(RescoreArgs a) {
    __shared__ float sc[kMaxLevels];
    load_centroids(sc, a.centroids, a.P.levels);
    const int m = *a.m_dev;
    const int D = a.P.D, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < m; row += gridDim.x * wpb) {
        const float *q = a.q_rot + (size_t)row * D, *s = a.s_q + (size_t)row * D;
        const float qn2 = a.norms[2 * row], qn = a.norms[2 * row + 1];
        float ad = INFINITY, ed = INFINITY;
        int ci = kNoIdx;
        if (lane < a.kc) {
            const long long id = a.cand_i[(size_t)row * a.kc + lane];
            if (id >= 0 && (size_t)id < a.n) {
                ci = (int)id;
                ad = a.cand_d[(size_t)row * a.kc + lane];
                ed = exact_dist<NIBBLE>(a.P, sc, q, s, qn2, qn, a.codes + (size_t)ci * a.P.cs, a.al4);
            }
        }
        float sq = 0.0f, ss = 0.0f;
        for (int i = lane; i < D; i += 32) {
            sq += fabsf(q[i]);
            ss += fabsf(s[i]);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            sq += __shfl_xor_sync(kFull, sq, off);
            ss += __shfl_xor_sync(kFull, ss, off);
        }
        // eps for this pass's candidates; eps_t for the threshold pass that may
        // rescan an open row (its own kappa, kappa_t >= kappa)
        const float terms = a.cmax * a.bound[0] * sq + a.bound[1] * ss;
        const float rest = 2.0f * qn * kDegenerateG * ss * a.bound[3] + kKappaEpi * (qn2 + a.bound[2]);
        const float eps = a.bound_scale * (2.0f * qn * a.kappa * terms + rest);
        const float eps_t = a.bound_scale * (2.0f * qn * a.kappa_t * terms + rest);
        const bool viol = ci != kNoIdx && !(fabsf(ad - ed) <= eps);
        const unsigned viol_mask = __ballot_sync(kFull, viol);
        const float ad_last = __shfl_sync(kFull, ad, a.kc - 1);
        const int ci_last = __shfl_sync(kFull, ci, a.kc - 1);
        // ascending bitonic sort of the 32 (exact distance, index) pairs
        float d = ed;
        int ix = ci;
#pragma unroll
        for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                const float od = __shfl_xor_sync(kFull, d, stride);
                const int ox = __shfl_xor_sync(kFull, ix, stride);
                const bool keep_min = (((lane & size) == 0) == ((lane & stride) == 0));
                const bool take = keep_min ? better(od, ox, d, ix) : better(d, ix, od, ox);
                if (take) {
                    d = od;
                    ix = ox;
                }
            }
        }
        const float ek = __shfl_sync(kFull, d, a.k - 1);
        // fewer than kc codes in the corpus: every code is a candidate
        const bool all_in = ci_last == kNoIdx;
        const bool certified = viol_mask == 0u && (all_in || ek < ad_last - eps);
        if (certified) {
            if (lane < a.k) {
                a.out_d[(size_t)row * a.k + lane] = d;
                a.out_i[(size_t)row * a.k + lane] = ix == kNoIdx ? -1 : (long long)ix;
            }
        } else if (lane == 0) {
            const int pos = atomicAdd(&a.counters[kCntFallbackRows], 1);
            a.fail_rows[pos] = row;
            a.thr[pos] = ek;
            a.tthr[pos] = viol_mask ? -1.0f : __fadd_ru(ek, eps_t);
            if (viol_mask) atomicAdd(&a.counters[kCntBoundViolations], __popc(viol_mask));
        }
    }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// distSearchScalarB4 in the reference build's order for D >= 64 (nb a
// multiple of 32), from per-query tables of its per-byte terms:
//   tip[b * 64 + (lo >> 1) + 8 (hi >> 1)] = fma(q[2b], c[lo >> 1], q[2b+1] * c[hi >> 1]),
//   tsg[b * 4 + (lo & 1) + 2 (hi & 1)]    = (+-s[2b]) + (+-s[2b+1]),
// the same FP32 operations as exact_b4 performs per byte, done once per query
// instead of once per code.  The running sums then take one table value per
// byte, in the same order.  code: 4-byte aligned.
__device__ __forceinline__ float exact_b4_tab(const float *__restrict__ tip,
                                              const float *__restrict__ tsg, float qn2, float qn,
                                              float scale, int nb, const uint8_t *code) {
    float A[32], S[32];
#pragma unroll
    for (int t = 0; t < 32; ++t) A[t] = S[t] = 0.0f;
#pragma unroll 1
    for (int b0 = 0; b0 < nb; b0 += 32) {
        const float *ti = tip + (size_t)b0 * 64, *ts = tsg + b0 * 4;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint32_t x = *reinterpret_cast<const uint32_t *>(code + b0 + 4 * w);
            // per byte: (lo >> 1) | (hi >> 1) << 3, and (lo & 1) | (hi & 1) << 1
            const uint32_t iw = ((x >> 1) & 0x07070707u) | ((x >> 2) & 0x38383838u);
            const uint32_t sw = (x & 0x01010101u) | ((x >> 3) & 0x02020202u);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int t = 4 * w + e;
                A[t] = __fadd_rn(A[t], ti[t * 64 + ((iw >> (8 * e)) & 0xFFu)]);
                S[t] = __fadd_rn(S[t], ts[t * 4 + ((sw >> (8 * e)) & 0xFFu)]);
            }
        }
    }
    float V[8], W[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        V[j] = __fadd_rn(__fadd_rn(A[16 + j], A[24 + j]), __fadd_rn(A[j], A[8 + j]));
        W[j] = __fadd_rn(__fadd_rn(S[16 + j], S[24 + j]), __fadd_rn(S[j], S[8 + j]));
    }
    const float ip = hsum8(V), dot = hsum8(W);
    const float xn = ld_f32(code + nb, true), g = ld_f32(code + nb + 4, true);
    const float sig = ld_f32(code + nb + 8, true);
    float t = __fmul_rn(__fmul_rn(scale, g), dot);
    t = __fmul_rn(__fmaf_rn(ip, sig, t), xn);
    return finish_dist(t, xn, qn2, qn);
}

struct CollectArgs {
    Params P;
    const float *centroids;
    const float *q_rot, *s_q, *norms;
    const uint8_t *codes;
    size_t n;
    bool al16;  // codes 16-byte aligned
    const int *fail_rows, *scan_rows, *counters;
    const float *thr;
    int *coll_n;
    float *coll_d;
    int *coll_i;
};

// The exact scan of the fallback.  For each of its rows g in turn (fail-list
// position f = scan_rows[g]), every CTA builds the row's term tables (TAB) in
// shared memory, then streams its share of the codes through two
// shared-memory chunk buffers (16-byte cp.async, the next chunk in flight
// while this one is scored), a thread per code.  A code whose exact distance
// is at most thr[f] is appended to the row's collection g (one atomic per
// warp).
template <bool NIBBLE, bool TAB>
__global__ void __launch_bounds__(256, 1) fallback_collect_kernel(CollectArgs a, int chunk,
                                                                  int tab_bytes) {
    const int ng = a.counters[kCntScanRows];
    if (ng == 0) return;
    extern __shared__ __align__(16) unsigned char fsm[];
    __shared__ float sc[kMaxLevels];
    load_centroids(sc, a.centroids, a.P.levels);
    const int D = a.P.D, nb = a.P.pb, cs = a.P.cs, lane = threadIdx.x & 31;
    const bool al4 = (cs & 3) == 0;
    float *tip = reinterpret_cast<float *>(fsm);
    float *tsg = tip + (size_t)nb * 64;
    unsigned char *cbuf = fsm + tab_bytes;
    const size_t cbytes = (size_t)chunk * cs, stride = (size_t)gridDim.x * chunk;
    auto stage = [&](int bsel, size_t c0) {
        const size_t rows = a.n - c0 < (size_t)chunk ? a.n - c0 : (size_t)chunk;
        const size_t bytes = rows * cs;
        const uint8_t *src = a.codes + c0 * cs;
        unsigned char *dst = cbuf + bsel * cbytes;
        size_t done = 0;
        if (a.al16) {
            const size_t n16 = bytes >> 4;
            for (size_t i = threadIdx.x; i < n16; i += blockDim.x) cp_async16(dst + 16 * i, src + 16 * i);
            done = n16 << 4;
        }
        for (size_t i = done + threadIdx.x; i < bytes; i += blockDim.x) dst[i] = src[i];
        cp_async_commit();
    };
    for (int g = 0; g < ng; ++g) {
        const int f = a.scan_rows[g];
        const int row = a.fail_rows[f];
        const float T = a.thr[f];
        const float *q = a.q_rot + (size_t)row * D, *s = a.s_q + (size_t)row * D;
        const float qn2 = a.norms[2 * row], qn = a.norms[2 * row + 1];
        __syncthreads();  // the previous row's tables and chunks are no longer read
        if constexpr (TAB) {
            for (int e = threadIdx.x; e < nb * 64; e += blockDim.x) {
                const int b = e >> 6;
                tip[e] = __fmaf_rn(q[2 * b], sc[e & 7], __fmul_rn(q[2 * b + 1], sc[(e >> 3) & 7]));
            }
            for (int e = threadIdx.x; e < nb * 4; e += blockDim.x) {
                const int b = e >> 2;
                tsg[e] = __fadd_rn(sgn_s(s[2 * b], e & 1), sgn_s(s[2 * b + 1], (e >> 1) & 1));
            }
        }
        size_t c0 = (size_t)blockIdx.x * chunk;
        int bsel = 0;
        if (c0 < a.n) stage(0, c0);
        for (; c0 < a.n; c0 += stride, bsel ^= 1) {
            if (c0 + stride < a.n)
                stage(bsel ^ 1, c0 + stride);
            else
                cp_async_commit();
            cp_async_wait1();
            __syncthreads();  // chunk c0 (and the tables) visible to every thread
            const int rows = (int)(a.n - c0 < (size_t)chunk ? a.n - c0 : (size_t)chunk);
            const int rows32 = (rows + 31) & ~31;
            const unsigned char *cb = cbuf + bsel * cbytes;
            for (int i = threadIdx.x; i < rows32; i += blockDim.x) {
                float d = 0.0f;
                bool pass = false;
                if (i < rows) {
                    const uint8_t *code = cb + (size_t)i * cs;
                    if constexpr (TAB)
                        d = exact_b4_tab(tip, tsg, qn2, qn, a.P.scale, nb, code);
                    else
                        d = exact_dist<NIBBLE>(a.P, sc, q, s, qn2, qn, code, al4);
                    pass = d <= T;
                }
                const unsigned m = __ballot_sync(kFull, pass);
                if (m) {
                    const int leader = __ffs(m) - 1;
                    int base = 0;
                    if (lane == leader) base = atomicAdd(&a.coll_n[g], __popc(m));
                    base = __shfl_sync(kFull, base, leader);
                    const int pos = base + __popc(m & ((1u << lane) - 1u));
                    if (pass && pos < kCollectCap) {
                        a.coll_d[(size_t)g * kCollectCap + pos] = d;
                        a.coll_i[(size_t)g * kCollectCap + pos] = (int)(c0 + (size_t)i);
                    }
                }
            }
            __syncthreads();  // buffer bsel is free for the chunk after next
        }
    }
}

// One warp per exact-scan row: the k best collected codes by (distance,
// index) to the output; a row whose collection overflowed (or that the scan
// could not take, collected == false) goes to the list pass's rows.
__global__ void __launch_bounds__(256) fallback_select_kernel(int *counters, const int *fail_rows,
                                                              const int *scan_rows, int k,
                                                              bool collected,
                                                              const int *__restrict__ coll_n,
                                                              const float *__restrict__ coll_d,
                                                              const int *__restrict__ coll_i,
                                                              int *list_rows, float *out_d,
                                                              long long *out_i) {
    const int ng = counters[kCntScanRows];
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int f = blockIdx.x * wpb + (threadIdx.x >> 5); f < ng; f += gridDim.x * wpb) {
        const int row = fail_rows[scan_rows[f]];
        const int cnt = coll_n[f];
        if (!collected || cnt > kCollectCap) {
            if (lane == 0) list_rows[atomicAdd(&counters[kCntListRows], 1)] = row;
            continue;
        }
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int u = 0; u < kTopKMax; ++u) {
            bd[u] = INFINITY;
            bi[u] = kNoIdx;
        }
        float td = INFINITY;
        int ti = kNoIdx;
        for (int u = lane; u < cnt; u += 32) {
            const float d = coll_d[(size_t)f * kCollectCap + u];
            const int i = coll_i[(size_t)f * kCollectCap + u];
            if (better(d, i, td, ti)) list_insert(bd, bi, k, d, i, &td, &ti);
        }
        float md;
        int mi;
        warp_merge(bd, bi, k, lane, md, mi);
        if (lane < k) {
            out_d[(size_t)row * k + lane] = md;
            out_i[(size_t)row * k + lane] = mi == kNoIdx ? -1 : (long long)mi;
        }
    }
}

// Tier 1: one warp per open row f.  When the tensor-core threshold pass ran
// (more than kTensorTierMinRows open rows), its bound held (tthr >= 0) and its
// list did not overflow, the lanes score the listed codes with the
// reference's arithmetic and the row's k best by (distance, index) go to the
// output.  The list holds the row's k best candidates (exact distance <= e_k)
// whenever the bound holds for them, so a k-th distance above e_k means it
// did not: that row, like every other, goes to the exact scan's rows.
template <bool NIBBLE>
__global__ void __launch_bounds__(256) tensor_select_kernel(
    Params P, const float *centroids, const float *q_rot, const float *s_q, const float *norms,
    const uint8_t *codes, size_t n, bool al4, int *counters, const int *fail_rows,
    const float *thr, const float *tthr, bool tensor_pass, int k, const int *__restrict__ coll_n,
    const int *__restrict__ coll_i, int *scan_rows, float *out_d, long long *out_i) {
    const int nf = counters[kCntFallbackRows];
    if (nf == 0) return;
    __shared__ float sc[kMaxLevels];
    load_centroids(sc, centroids, P.levels);
    const int D = P.D, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const bool ran = tensor_pass && nf > kTensorTierMinRows;
    for (int f = blockIdx.x * wpb + (threadIdx.x >> 5); f < nf; f += gridDim.x * wpb) {
        const int cnt = coll_n[f];
        if (!ran || !(tthr[f] >= 0.0f) || cnt > kCollectCap) {
            if (lane == 0) scan_rows[atomicAdd(&counters[kCntScanRows], 1)] = f;
            continue;
        }
        const int row = fail_rows[f];
        const float *q = q_rot + (size_t)row * D, *s = s_q + (size_t)row * D;
        const float qn2 = norms[2 * row], qn = norms[2 * row + 1];
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int u = 0; u < kTopKMax; ++u) {
            bd[u] = INFINITY;
            bi[u] = kNoIdx;
        }
        float td = INFINITY;
        int ti = kNoIdx;
        for (int u = lane; u < cnt; u += 32) {
            const int j = coll_i[(size_t)f * kCollectCap + u];
            if (j < 0 || (size_t)j >= n) continue;
            const float d = exact_dist<NIBBLE>(P, sc, q, s, qn2, qn, codes + (size_t)j * P.cs, al4);
            if (better(d, j, td, ti)) list_insert(bd, bi, k, d, j, &td, &ti);
        }
        float md;
        int mi;
        warp_merge(bd, bi, k, lane, md, mi);
        const float kth = __shfl_sync(kFull, md, k - 1);
        if (!(kth <= thr[f])) {
            if (lane == 0) scan_rows[atomicAdd(&counters[kCntScanRows], 1)] = f;
            continue;
        }
        if (lane < k) {
            out_d[(size_t)row * k + lane] = md;
            out_i[(size_t)row * k + lane] = mi == kNoIdx ? -1 : (long long)mi;
        }
    }
}

// Open row f's query planes (K BF16 values a row, hi and lo) and scales to
// row f of the tensor-core threshold pass's operands.
__global__ void __launch_bounds__(256) gather_open_kernel(const int *__restrict__ counters,
                                                          const int *__restrict__ fail_rows,
                                                          const uint4 *__restrict__ ah,
                                                          const uint4 *__restrict__ al,
                                                          const float *__restrict__ r1,
                                                          const float *__restrict__ r2, int w16,
                                                          uint4 *__restrict__ ah2,
                                                          uint4 *__restrict__ al2,
                                                          float *__restrict__ r1o,
                                                          float *__restrict__ r2o) {
    const int nf = counters[kCntFallbackRows];
    if (nf <= kTensorTierMinRows) return;
    const size_t total = (size_t)nf * w16;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t f = t / w16, w = t % w16;
        const size_t src = (size_t)fail_rows[f] * w16 + w;
        ah2[t] = ah[src];
        al2[t] = al[src];
        if (w == 0) {
            r1o[f] = r1[fail_rows[f]];
            r2o[f] = r2[fail_rows[f]];
        }
    }
}

struct FallbackArgs {
    Params P;
    const float *centroids;
    int k;
    const float *q_rot, *s_q, *norms;
    const uint8_t *codes;
    size_t n;
    bool al16;  // codes 16-byte aligned
    const int *rows, *counters;
    float *part_d;
    int *part_i;
};

// The list pass for the rows the exact scan could not settle
// (counters[kCntListRows] of them, in rows): a full pass over the codes
// for each row.  A CTA stages chunks of `chunk` consecutive codes in shared
// memory with coalesced 16-byte loads, then each thread scores the codes of
// the chunk it owns from there (a code's words are cs / 4 apart, an odd
// stride: no bank conflicts) and keeps a sorted list; the warps merge their
// lanes' lists and warp 0 merges the block's into part[row][cta].
template <bool NIBBLE>
__global__ void __launch_bounds__(256) fallback_scan_kernel(FallbackArgs a, int chunk) {
    const int nf = a.counters[kCntListRows];
    if (nf == 0) return;
    extern __shared__ __align__(16) unsigned char fsm[];
    __shared__ float sc[kMaxLevels];
    __shared__ float wd[8][kTopKMax];
    __shared__ int wi[8][kTopKMax];
    load_centroids(sc, a.centroids, a.P.levels);
    const int D = a.P.D, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int k = a.k, cs = a.P.cs;
    const bool al4 = (cs & 3) == 0;
    for (int f = 0; f < nf; ++f) {
        const int row = a.rows[f];
        const float *q = a.q_rot + (size_t)row * D, *s = a.s_q + (size_t)row * D;
        const float qn2 = a.norms[2 * row], qn = a.norms[2 * row + 1];
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int u = 0; u < kTopKMax; ++u) {
            bd[u] = INFINITY;
            bi[u] = kNoIdx;
        }
        float td = INFINITY;
        int ti = kNoIdx;
        for (size_t c0 = (size_t)blockIdx.x * chunk; c0 < a.n; c0 += (size_t)gridDim.x * chunk) {
            const int rows = (int)(a.n - c0 < (size_t)chunk ? a.n - c0 : (size_t)chunk);
            const size_t bytes = (size_t)rows * cs;
            const uint8_t *src = a.codes + c0 * cs;
            __syncthreads();  // the previous chunk is scored
            if (a.al16) {
                const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
                uint4 *d4 = reinterpret_cast<uint4 *>(fsm);
                for (size_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d4[i] = __ldg(s4 + i);
                for (size_t i = (bytes & ~size_t(15)) + threadIdx.x; i < bytes; i += blockDim.x) fsm[i] = src[i];
            } else {
                for (size_t i = threadIdx.x; i < bytes; i += blockDim.x) fsm[i] = src[i];
            }
            __syncthreads();
            for (int i = threadIdx.x; i < rows; i += blockDim.x) {
                const int j = (int)(c0 + (size_t)i);
                const float d = exact_dist<NIBBLE>(a.P, sc, q, s, qn2, qn, fsm + (size_t)i * cs, al4);
                if (better(d, j, td, ti)) list_insert(bd, bi, k, d, j, &td, &ti);
            }
        }
        float md;
        int mi;
        warp_merge(bd, bi, k, lane, md, mi);
        if (lane < k) {
            wd[warp][lane] = md;
            wi[warp][lane] = mi;
        }
        __syncthreads();
        if (warp == 0) {
            float ld[kTopKMax];
            int li[kTopKMax];
#pragma unroll
            for (int u = 0; u < kTopKMax; ++u) {
                ld[u] = (lane < nw && u < k) ? wd[lane][u] : INFINITY;
                li[u] = (lane < nw && u < k) ? wi[lane][u] : kNoIdx;
            }
            warp_merge(ld, li, k, lane, md, mi);
            if (lane < k) {
                const size_t o = ((size_t)f * gridDim.x + blockIdx.x) * k + lane;
                a.part_d[o] = md;
                a.part_i[o] = mi;
            }
        }
        __syncthreads();
    }
}

// One warp per list-pass row: merge the CTAs' lists into the row's output.
__global__ void __launch_bounds__(256) fallback_merge_kernel(const int *__restrict__ counters,
                                                             const int *__restrict__ rows, int ctas,
                                                             int k, const float *__restrict__ part_d,
                                                             const int *__restrict__ part_i,
                                                             float *__restrict__ out_d,
                                                             long long *__restrict__ out_i) {
    const int nf = counters[kCntListRows];
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int f = blockIdx.x * wpb + (threadIdx.x >> 5); f < nf; f += gridDim.x * wpb) {
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int u = 0; u < kTopKMax; ++u) {
            bd[u] = INFINITY;
            bi[u] = kNoIdx;
        }
        float td = INFINITY;
        int ti = kNoIdx;
        for (int c = lane; c < ctas; c += 32)
            for (int u = 0; u < k; ++u) {
                const size_t o = ((size_t)f * ctas + c) * k + u;
                const float d = part_d[o];
                const int i = part_i[o];
                if (i != kNoIdx && better(d, i, td, ti)) list_insert(bd, bi, k, d, i, &td, &ti);
            }
        float md;
        int mi;
        warp_merge(bd, bi, k, lane, md, mi);
        const int row = rows[f];
        if (lane < k) {
            out_d[(size_t)row * k + lane] = md;
            out_i[(size_t)row * k + lane] = mi == kNoIdx ? -1 : (long long)mi;
        }
    }
}

template <bool NIBBLE>
__global__ void __launch_bounds__(256) exact_mton_kernel(Params P, const float *centroids,
                                                         const float *q_rot, const float *s_q,
                                                         const float *norms, size_t m,
                                                         const uint8_t *codes, size_t n, bool al4,
                                                         float *out, size_t ldo) {
    __shared__ float sc[kMaxLevels];
    load_centroids(sc, centroids, P.levels);
    const size_t total = m * n;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / n, j = t % n;
        out[r * ldo + j] = exact_dist<NIBBLE>(P, sc, q_rot + r * P.D, s_q + r * P.D, norms[2 * r],
                                    norms[2 * r + 1], codes + j * P.cs, al4);
    }
}

// The reference build's symmetric distance of codes a and b
// (distBuildAVX :1541-1612 / distBuildScalarB4 :985-1019 as its compiler
// vectorised them), in that build's own summation order:
//   byte codes, D >= 8: 8 running sums fma(c_a c_b, sigma_a sigma_b, S[i mod 8]),
//     folded as hsum8; D < 8: one sum in coordinate order;
//   nibble codes, with pair(f, k0, k1) = fma(f_a(k0), f_b(k0), f_a(k1) f_b(k1)):
//     blocks of 32 bytes k, lanes j < 8:
//       s = ((pair(hi, k+16+j, k+24+j) + pair(hi, k+j, k+8+j)) + pair(lo, k+j, k+8+j))
//           + pair(lo, k+16+j, k+24+j),  S[j] = fma(s sigma_a, sigma_b, S[j]), hsum8;
//     16 bytes (D = 32): 4 lanes, offsets 4 / 8 / 12, S[j] = (s sigma_a) sigma_b, hsum4;
//     <= 8 bytes: ip = fma(fma(lo_a, lo_b, hi_a hi_b), sigma_a sigma_b, ip) in byte order;
//   d = max(0, fma(-(ip + ip), |a| |b|, fma(|a|, |a|, |b| |b|))).
template <bool NIBBLE>
__device__ float exact_sym_dist(const Params &P, const float *sc, const uint8_t *a, const uint8_t *b,
                                bool al4) {
    const int nb = P.pb;
    const float na = ld_f32(a + nb, al4), sa = ld_f32(a + nb + 8, al4);
    const float nbn = ld_f32(b + nb, al4), sb = ld_f32(b + nb + 8, al4);
    const float sab = __fmul_rn(sa, sb);
    float ip = 0.0f;
    if constexpr (!NIBBLE) {
        const int D = P.D;
        int i = 0;
        if (D >= 8) {
            float S[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            for (; i + 8 <= D; i += 8)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    S[j] = __fmaf_rn(__fmul_rn(sc[a[i + j] >> 1], sc[b[i + j] >> 1]), sab, S[j]);
            ip = hsum8(S);
        }
        for (; i < D; ++i) ip = __fmaf_rn(__fmul_rn(sc[a[i] >> 1], sc[b[i] >> 1]), sab, ip);
    } else {
        auto lo = [&](const uint8_t *x, int k) { return sc[(x[k] & 15u) >> 1]; };
        auto hi = [&](const uint8_t *x, int k) { return sc[(x[k] >> 4) >> 1]; };
        auto pair_lo = [&](int k0, int k1) {
            return __fmaf_rn(lo(a, k0), lo(b, k0), __fmul_rn(lo(a, k1), lo(b, k1)));
        };
        auto pair_hi = [&](int k0, int k1) {
            return __fmaf_rn(hi(a, k0), hi(b, k0), __fmul_rn(hi(a, k1), hi(b, k1)));
        };
        int k = 0;
        if (nb >= 32) {
            float S[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            for (; k + 32 <= nb; k += 32)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int l0 = k + j, l1 = l0 + 16;
                    const float s = __fadd_rn(__fadd_rn(__fadd_rn(pair_hi(l1, l1 + 8), pair_hi(l0, l0 + 8)),
                                                        pair_lo(l0, l0 + 8)),
                                              pair_lo(l1, l1 + 8));
                    S[j] = __fmaf_rn(__fmul_rn(s, sa), sb, S[j]);
                }
            ip = hsum8(S);
        }
        if (nb - k >= 16) {
            float S4[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int l0 = k + j, l1 = l0 + 8;
                const float s = __fadd_rn(__fadd_rn(__fadd_rn(pair_hi(l1, l1 + 4), pair_hi(l0, l0 + 4)),
                                                    pair_lo(l0, l0 + 4)),
                                          pair_lo(l1, l1 + 4));
                S4[j] = __fmul_rn(__fmul_rn(s, sa), sb);
            }
            ip = __fadd_rn(ip, hsum4(S4));
            k += 16;
        }
        for (; k < nb; ++k)
            ip = __fmaf_rn(__fmaf_rn(lo(a, k), lo(b, k), __fmul_rn(hi(a, k), hi(b, k))), sab, ip);
    }
    const float d = __fmaf_rn(-__fadd_rn(ip, ip), __fmul_rn(na, nbn), __fmaf_rn(na, na, __fmul_rn(nbn, nbn)));
    return 0.0f < d ? d : 0.0f;
}

// Symmetric distances of m codes A against n codes B in the reference build's
// order: one thread per pair.
template <bool NIBBLE>
__global__ void __launch_bounds__(256) exact_sym_kernel(Params P, const float *centroids,
                                                        const uint8_t *A, size_t m, const uint8_t *B,
                                                        size_t n, bool al4, float *out, size_t ldo) {
    __shared__ float sc[kMaxLevels];
    load_centroids(sc, centroids, P.levels);
    const size_t total = m * n;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / n, j = t % n;
        out[r * ldo + j] = exact_sym_dist<NIBBLE>(P, sc, A + r * P.cs, B + j * P.cs, al4);
    }
}

// Index-wide maxima of sigma |x|, scale gamma |x|, |x|^2 and |x| (bound must
// be zeroed; non-negative floats order like their bit patterns, NaN counts as
// +inf).
__global__ void __launch_bounds__(256) index_bound_kernel(Params P, const uint8_t *codes, size_t n,
                                                          float *bound) {
    float v[kBoundFloats] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (size_t)gridDim.x * blockDim.x) {
        const uint8_t *t = codes + j * P.cs + P.pb;
        const bool al4 = ((reinterpret_cast<uintptr_t>(t) & 3) == 0);
        const float xn = fabsf(ld_f32(t, al4)), g = fabsf(ld_f32(t + 4, al4));
        const float sig = fabsf(ld_f32(t + 8, al4));
        const float w[kBoundFloats] = {sig * xn, P.scale * g * xn, xn * xn, xn};
#pragma unroll
        for (int i = 0; i < kBoundFloats; ++i) v[i] = (w[i] != w[i]) ? INFINITY : fmaxf(v[i], w[i]);
    }
#pragma unroll
    for (int i = 0; i < kBoundFloats; ++i) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[i] = fmaxf(v[i], __shfl_xor_sync(kFull, v[i], off));
        if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(bound) + i, __float_as_int(v[i]));
    }
}

// Batch row r of the serving path <- pool row rows[r] (r < *m_dev).
__global__ void __launch_bounds__(256) gather_rows_kernel(const float *__restrict__ pool,
                                                          const int *__restrict__ rows,
                                                          const int *__restrict__ m_dev, int dim,
                                                          float *__restrict__ out) {
    const int m = *m_dev;
    const size_t total = (size_t)m * dim;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / dim, i = t % dim;
        out[t] = pool[(size_t)rows[r] * dim + i];
    }
}

bool codes_al4(const Params &P, const uint8_t *codes) {
    return (P.cs % 4 == 0) && ((reinterpret_cast<uintptr_t>(codes) & 3) == 0);
}

}  // namespace

cudaError_t launch_index_bound(const Params &P, const uint8_t *codes, size_t n, float *bound,
                               cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(bound, 0, kBoundFloats * sizeof(float), st);
    if (e != cudaSuccess || n == 0) return e;
    const size_t blocks = std::min<size_t>((n + 255) / 256, 4096);
    index_bound_kernel<<<(unsigned)blocks, 256, 0, st>>>(P, codes, n, bound);
    return cudaGetLastError();
}

cudaError_t launch_rescore(const Params &P, const float *centroids, float cmax, const int *m_dev,
                           int kc, int k, const float *cand_d, const long long *cand_i,
                           const float *q_rot, const float *s_q, const float *norms,
                           const uint8_t *codes, size_t n, const float *bound, float kappa,
                           float kappa_t, float bound_scale,
                           float *out_d, long long *out_i, int *fail_rows, float *thr, float *tthr,
                           int *counters, int max_rows, cudaStream_t st) {
    if (kc < 1 || kc > 32 || k < 1 || k > kc || k > kTopKMax || max_rows < 1 || !(kappa > 0.0f))
        return cudaErrorInvalidValue;
    const RescoreArgs a{P,     centroids, cmax,  m_dev,     kc,          k,     cand_d,
                        cand_i, q_rot,    s_q,   norms,     codes,       n,     codes_al4(P, codes),
                        bound, kappa, kappa_t > kappa ? kappa_t : kappa, bound_scale, out_d, out_i,
                        fail_rows, thr, tthr, counters};
    const unsigned blocks = (unsigned)((max_rows + 7) / 8);
    if (P.nibble)
        rescore_kernel<true><<<blocks, 256, 0, st>>>(a);
    else
        rescore_kernel<false><<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

int fallback_ctas(int sms) { return 2 * (sms > 0 ? sms : 148); }

cudaError_t launch_gather_open(const int *counters, const int *fail_rows, const void *ah,
                               const void *al, const float *r1, const float *r2, int K,
                               int max_rows, void *ah2, void *al2, float *r1o, float *r2o,
                               cudaStream_t st) {
    if (K % 8 || max_rows < 1) return cudaErrorInvalidValue;
    const uintptr_t any = reinterpret_cast<uintptr_t>(ah) | reinterpret_cast<uintptr_t>(al) |
                          reinterpret_cast<uintptr_t>(ah2) | reinterpret_cast<uintptr_t>(al2);
    if (any & 15) return cudaErrorMisalignedAddress;
    const int w16 = K / 8;  // 16-byte words of a BF16 row
    const size_t total = (size_t)max_rows * w16;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 4);
    gather_open_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(
        counters, fail_rows, static_cast<const uint4 *>(ah), static_cast<const uint4 *>(al), r1, r2,
        w16, static_cast<uint4 *>(ah2), static_cast<uint4 *>(al2), r1o, r2o);
    return cudaGetLastError();
}

cudaError_t launch_fallback(const Params &P, const float *centroids, int k, const float *q_rot,
                            const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                            const int *fail_rows, int *counters, int fb_ctas, bool tensor_pass,
                            const FallbackBuffers &fb, float *out_d, long long *out_i,
                            int max_rows, cudaStream_t st) {
    if (k < 1 || k > kTopKMax || fb_ctas < 1 || max_rows < 1) return cudaErrorInvalidValue;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const unsigned rblocks = (unsigned)((max_rows + 7) / 8);
    int *scan_n = fb.coll_n + max_rows;
    // tier 1: the tensor-core pass's lists (coll_n[0..R) was zeroed before it)
    if (P.nibble)
        tensor_select_kernel<true><<<rblocks, 256, 0, st>>>(
            P, centroids, q_rot, s_q, norms, codes, n, codes_al4(P, codes), counters, fail_rows,
            fb.thr, fb.tthr, tensor_pass, k, fb.coll_n, fb.coll_i, fb.scan_rows, out_d, out_i);
    else
        tensor_select_kernel<false><<<rblocks, 256, 0, st>>>(
            P, centroids, q_rot, s_q, norms, codes, n, codes_al4(P, codes), counters, fail_rows,
            fb.thr, fb.tthr, tensor_pass, k, fb.coll_n, fb.coll_i, fb.scan_rows, out_d, out_i);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // tier 2: the exact scan.  Chunks start at code indices that are multiples
    // of 16: 16-byte aligned with the base.
    const bool al16 = (reinterpret_cast<uintptr_t>(codes) & 15) == 0;
    constexpr int kThreads = 256;
    constexpr size_t kSmemMax = 224 * 1024;
    // term tables when nibble codes have D >= 64 and the tables leave room for
    // two chunks of at least 16 codes
    const size_t cs = (size_t)P.cs;
    const size_t tab_bytes = (size_t)P.pb * (64 + 4) * 4;
    const bool tab = P.nibble && P.D >= 64 && P.pb % 32 == 0 && tab_bytes + 32 * cs <= kSmemMax;
    const size_t tb = tab ? tab_bytes : 0;
    const int chunk = (int)std::min<size_t>(256, (kSmemMax - std::min(tb, kSmemMax)) / (2 * cs)) & ~15;
    const bool collected = chunk >= 16 && (cs & 3) == 0;
    e = cudaMemsetAsync(scan_n, 0, (size_t)max_rows * sizeof(int), st);
    if (e != cudaSuccess) return e;
    if (collected) {
        const CollectArgs ca{P,         centroids,    q_rot,    s_q,    norms,  codes,     n,
                             al16,      fail_rows,    fb.scan_rows, counters, fb.thr, scan_n,
                             fb.coll_d, fb.coll_i};
        const size_t smem = tb + 2 * (size_t)chunk * cs;
        auto kern = !P.nibble ? fallback_collect_kernel<false, false>
                              : (tab ? fallback_collect_kernel<true, true> : fallback_collect_kernel<true, false>);
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
        if (e != cudaSuccess) return e;
        const int grid = std::max(1, per_sm) * std::max(1, sms);
        kern<<<grid, kThreads, smem, st>>>(ca, chunk, (int)tb);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    fallback_select_kernel<<<rblocks, 256, 0, st>>>(counters, fail_rows, fb.scan_rows, k, collected,
                                                    scan_n, fb.coll_d, fb.coll_i, fb.list_rows,
                                                    out_d, out_i);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // tier 3: the list pass.  Codes per staged chunk up to 256, at most 96 KB
    // of shared memory, a multiple of 16 so that every chunk starts 16-byte
    // aligned.
    const FallbackArgs a{P,  centroids, k, q_rot, s_q, norms, codes, n, al16, fb.list_rows, counters,
                         fb.part_d, fb.part_i};
    int lchunk = (int)std::min<size_t>(256, (size_t)(96 * 1024) / cs) & ~15;
    if (lchunk < 16) lchunk = 16;
    const size_t lsmem = (size_t)lchunk * cs;
    auto lkern = P.nibble ? fallback_scan_kernel<true> : fallback_scan_kernel<false>;
    e = cudaFuncSetAttribute(lkern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem);
    if (e != cudaSuccess) return e;
    lkern<<<fb_ctas, 256, lsmem, st>>>(a, lchunk);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fallback_merge_kernel<<<rblocks, 256, 0, st>>>(counters, fb.list_rows, fb_ctas, k, fb.part_d,
                                                   fb.part_i, out_d, out_i);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float *pool, const int *rows, const int *m_dev, size_t dim,
                               size_t max_rows, float *out, cudaStream_t st) {
    const size_t total = max_rows * dim;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 8);
    gather_rows_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(pool, rows, m_dev, (int)dim, out);
    return cudaGetLastError();
}

cudaError_t launch_exact_mton(const Params &P, const float *centroids, const float *q_rot,
                              const float *s_q, const float *norms, size_t m, const uint8_t *codes,
                              size_t n, float *out, size_t ldo, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    const size_t total = m * n;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
    if (P.nibble)
        exact_mton_kernel<true><<<blocks, 256, 0, st>>>(P, centroids, q_rot, s_q, norms, m, codes, n,
                                                        codes_al4(P, codes), out, ldo);
    else
        exact_mton_kernel<false><<<blocks, 256, 0, st>>>(P, centroids, q_rot, s_q, norms, m, codes, n,
                                                         codes_al4(P, codes), out, ldo);
    return cudaGetLastError();
}

cudaError_t launch_exact_mton_sym(const Params &P, const float *centroids, const uint8_t *A, size_t m,
                                  const uint8_t *B, size_t n, float *out, size_t ldo, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    const size_t total = m * n;
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
    const bool al4 = codes_al4(P, A) && codes_al4(P, B);
    if (P.nibble)
        exact_sym_kernel<true><<<blocks, 256, 0, st>>>(P, centroids, A, m, B, n, al4, out, ldo);
    else
        exact_sym_kernel<false><<<blocks, 256, 0, st>>>(P, centroids, A, m, B, n, al4, out, ldo);
    return cudaGetLastError();
}

}  // namespace tq
