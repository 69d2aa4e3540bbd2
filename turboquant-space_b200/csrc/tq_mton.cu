// tq_mton.cu -- the M x N distance contractions (distanceBatchMToN and
// distanceBatchMToNSymmetric, space_turbo_quant.h:588-615) as dense GEMMs.
//
// Once a code is decoded to centroid values the distance is a contraction.
// Both sides are decoded into operand "planes" (row-major, K contiguous):
//
//   asymmetric, K = 2D:  A[i] = [ q_rot_i           | s_q_i                     ]
//                        B[j] = [ sigma_j c[idx_j]  | scale gamma_j (+-1)_j     ]
//                        so (A B^T)[i, j] = ip_mse + correction of distSearch
//                        (:676-683); r1 = |q|, r2 = |q|^2, c1 = |x|, c2 = |x|^2
//   symmetric,  K = D:   A[i] = c[idx_a_i], B[j] = c[idx_b_j]
//                        r1 = sigma_a n_a, r2 = n_a^2, c1 = sigma_b n_b, c2 = n_b^2
//                        (distBuild :707-713 with both sigmas factored out)
//
// and every result is d = max(0, r2_i + c2_j - 2 (C_ij r1_i) c1_j).
//
// Planes come in two formats: FP32 (the CUDA-core SGEMM below, the drop-in)
// and a hi/lo BF16 pair, x = hi + lo with hi = bf16(x), lo = bf16(x - hi),
// for the tcgen05 kernel (tq_tc.cu), which forms hi*hi + hi*lo + lo*hi.
//
// Asymmetric BF16 column planes use the exact-sign form: with g_j = scale
// gamma_j, B[j] = [ sigma_j c[idx_j] / g_j | (+-1)_j ] and c1 = g_j |x|, so
// the QJL half is exact in BF16 (its lo plane is zero and is not stored: the
// lo plane has asym_lo_width(D) columns) and the tensor-core kernel needs two
// products there instead of three.  A code with g_j < 1e-20 (gamma = 0, e.g.
// a zero row) keeps B[j] = [ sigma_j c[idx_j] | 0 ] and c1 = |x|: its
// correction term is below 1e-18 of |q| |x| and is left out.
#include <cuda_bf16.h>

#include <algorithm>

#include "tq_internal.h"
#include "tq_mton.h"

namespace tq {
namespace {

__device__ __forceinline__ unsigned unit_at(const uint8_t *code, int p, int nibble) {
    if (nibble) {
        const unsigned b = code[p >> 1];
        return (p & 1) ? (b >> 4) : (b & 15u);
    }
    return code[p];
}

// Value v at position k of row r: FP32 plane0[r K + k], or BF16 hi at
// plane0[r K + k] and lo at plane1[r ldl + k] (k < ldl; beyond ldl lo is zero
// by construction and not stored).
__device__ __forceinline__ void put(void *plane0, void *plane1, size_t r, int K, int ldl, int k,
                                    float v, int fmt) {
    if (fmt == kPlaneF32) {
        static_cast<float *>(plane0)[r * K + k] = v;
    } else {
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        static_cast<__nv_bfloat16 *>(plane0)[r * K + k] = hi;
        if (k < ldl)
            static_cast<__nv_bfloat16 *>(plane1)[r * ldl + k] =
                __float2bfloat16_rn(v - __bfloat162float(hi));
    }
}

// One thread per (row, 4 consecutive positions).  Rows in [rows, rows_pad)
// are zero so that padded tiles contribute nothing.
__global__ void __launch_bounds__(256) planes_from_codes_kernel(
    const uint8_t *__restrict__ codes, size_t rows, size_t rows_pad, Params P, DevTables T,
    int sym, int fmt, int ldl, void *plane0, void *plane1, float *__restrict__ s1,
    float *__restrict__ s2) {
    const int K = sym ? P.D : 2 * P.D;
    const bool exact_sign = !sym && fmt == kPlaneBF16;
    const size_t quads_per_row = (size_t)(K / 4);
    const size_t total = rows_pad * quads_per_row;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / quads_per_row;
        const int k0 = (int)(t - r * quads_per_row) * 4;
        if (r >= rows) {
            for (int q = 0; q < 4; ++q) put(plane0, plane1, r, K, ldl, k0 + q, 0.0f, fmt);
            if (k0 == 0) {
                s1[r] = 0.0f;
                s2[r] = 0.0f;
            }
            continue;
        }
        const uint8_t *code = codes + r * (size_t)P.cs;
        float meta[3];
        for (int q = 0; q < 3; ++q) {
            uint32_t w = 0;
            for (int b = 0; b < 4; ++b) w |= (uint32_t)code[P.pb + 4 * q + b] << (8 * b);
            meta[q] = __uint_as_float(w);
        }
        const float norm = meta[0], gamma = meta[1], sigma = meta[2];
        const float sg = __fmul_rn(P.scale, gamma);
        // exact-sign form: g = scale gamma factored out of the column (see the
        // file header); !(g >= 1e-20f) also catches a NaN trailer
        const bool ratio = exact_sign && sg >= 1e-20f && sg <= 3.0e38f;
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            float v;
            if (sym) {
                v = T.centroids[unit_at(code, k, P.nibble) >> 1];
            } else if (k < P.D) {
                v = __fmul_rn(sigma, T.centroids[unit_at(code, k, P.nibble) >> 1]);
                if (ratio) v = __fdiv_rn(v, sg);
            } else {
                const bool pos = unit_at(code, k - P.D, P.nibble) & 1u;
                if (!exact_sign) v = pos ? sg : -sg;
                else v = !ratio ? 0.0f : pos ? 1.0f : -1.0f;
            }
            put(plane0, plane1, r, K, ldl, k, v, fmt);
        }
        if (k0 == 0) {
            s1[r] = sym ? __fmul_rn(sigma, norm) : ratio ? __fmul_rn(sg, norm) : norm;
            s2[r] = __fmul_rn(norm, norm);
        }
    }
}

// Scalars of the decoded-B kernels (launch_dec_factors): the same per-code
// quantities as the planes' s1 / s2 and exact-sign ratio, with the ratio as a
// chunk factor instead of a division of every value.
__global__ void __launch_bounds__(256) dec_factors_kernel(const uint8_t *__restrict__ codes,
                                                          size_t rows, size_t rows_pad, Params P,
                                                          int sym, float *__restrict__ c1,
                                                          float *__restrict__ c2,
                                                          float *__restrict__ fc,
                                                          float *__restrict__ fs) {
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows_pad;
         r += (size_t)gridDim.x * blockDim.x) {
        float a = 0.0f, b = 0.0f, f = 0.0f, g1 = 0.0f;
        if (r < rows) {
            const uint8_t *t = codes + r * (size_t)P.cs + P.pb;
            float meta[3];
            for (int q = 0; q < 3; ++q) {
                uint32_t w = 0;
                for (int k = 0; k < 4; ++k) w |= (uint32_t)t[4 * q + k] << (8 * k);
                meta[q] = __uint_as_float(w);
            }
            const float norm = meta[0], gamma = meta[1], sigma = meta[2];
            b = __fmul_rn(norm, norm);
            if (sym) {
                a = __fmul_rn(sigma, norm);
            } else {
                const float sg = __fmul_rn(P.scale, gamma);
                const bool ratio = sg >= 1e-20f && sg <= 3.0e38f;  // as the exact-sign planes
                a = ratio ? __fmul_rn(sg, norm) : norm;
                f = ratio ? __fdiv_rn(sigma, sg) : sigma;
                g1 = ratio ? 1.0f : 0.0f;
            }
        }
        c1[r] = a;
        c2[r] = b;
        if (fc) fc[r] = f;
        if (fs) fs[r] = g1;
    }
}

__global__ void __launch_bounds__(256) planes_from_prepared_kernel(
    const float *__restrict__ q_rot, const float *__restrict__ s_q, const float *__restrict__ norms,
    size_t rows, size_t rows_pad, int D, int fmt, void *plane0, void *plane1,
    float *__restrict__ r1, float *__restrict__ r2) {
    const int K = 2 * D;
    const size_t total = rows_pad * (size_t)K;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / K;
        const int k = (int)(t - r * K);
        float v = 0.0f;
        if (r < rows) v = (k < D) ? q_rot[r * D + k] : s_q[r * D + (k - D)];
        put(plane0, plane1, r, K, K, k, v, fmt);
        if (k == 0) {
            r1[r] = (r < rows) ? norms[2 * r + 1] : 0.0f;
            r2[r] = (r < rows) ? norms[2 * r] : 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// FP32 CUDA-core GEMM with the distance epilogue: 128 x 128 tile, K step 16,
// 256 threads, 8 x 8 outputs per thread (two 4 x 4 quadrants 64 apart),
// double-buffered shared tiles stored K-major-transposed for float4 reads.
// The tile column is XOR-swizzled with bit 3 of k (sw_col), which keeps each
// float4 group intact and makes the transposed stores conflict-free.  Row
// blocks are blockIdx.x (fastest), so CTAs running together share the B tile
// in L2; two CTAs per SM.
// A: rows_pad(m) x K, B: rows_pad(n) x K, both multiples of 128 rows, K % 16 == 0.
// ---------------------------------------------------------------------------
constexpr int SG_BM = 128, SG_BN = 128, SG_BK = 16, SG_PAD = 4;

__device__ __forceinline__ int sw_col(int k, int col) { return col ^ (((k >> 3) & 1) << 3); }

__global__ void __launch_bounds__(256, 2) sgemm_dist_kernel(
    const float *__restrict__ A, const float *__restrict__ B, int K, size_t m, size_t n,
    const float *__restrict__ r1, const float *__restrict__ r2, const float *__restrict__ c1,
    const float *__restrict__ c2, float *__restrict__ out, size_t ldo) {
    __shared__ __align__(16) float As[2][SG_BK][SG_BM + SG_PAD];
    __shared__ __align__(16) float Bs[2][SG_BK][SG_BN + SG_PAD];
    const int tid = threadIdx.x;
    const size_t m0 = (size_t)blockIdx.x * SG_BM, n0 = (size_t)blockIdx.y * SG_BN;
    const int lrow = tid >> 2, lk = (tid & 3) * 4;
    const float *Ag = A + (m0 + lrow) * (size_t)K + lk;
    const float *Bg = B + (n0 + lrow) * (size_t)K + lk;
    const size_t half = (size_t)64 * K;
    float4 ra0, ra1, rb0, rb1;
    auto gload = [&](int kt) {
        const size_t o = (size_t)kt * SG_BK;
        ra0 = __ldg(reinterpret_cast<const float4 *>(Ag + o));
        ra1 = __ldg(reinterpret_cast<const float4 *>(Ag + half + o));
        rb0 = __ldg(reinterpret_cast<const float4 *>(Bg + o));
        rb1 = __ldg(reinterpret_cast<const float4 *>(Bg + half + o));
    };
    // lk + q has the same bit 3 for q < 4, so one swizzled column per thread
    const int r0s = sw_col(lk, lrow), r1s = sw_col(lk, lrow + 64);
    auto sstore = [&](int buf) {
        As[buf][lk + 0][r0s] = ra0.x; As[buf][lk + 1][r0s] = ra0.y;
        As[buf][lk + 2][r0s] = ra0.z; As[buf][lk + 3][r0s] = ra0.w;
        As[buf][lk + 0][r1s] = ra1.x; As[buf][lk + 1][r1s] = ra1.y;
        As[buf][lk + 2][r1s] = ra1.z; As[buf][lk + 3][r1s] = ra1.w;
        Bs[buf][lk + 0][r0s] = rb0.x; Bs[buf][lk + 1][r0s] = rb0.y;
        Bs[buf][lk + 2][r0s] = rb0.z; Bs[buf][lk + 3][r0s] = rb0.w;
        Bs[buf][lk + 0][r1s] = rb1.x; Bs[buf][lk + 1][r1s] = rb1.y;
        Bs[buf][lk + 2][r1s] = rb1.z; Bs[buf][lk + 3][r1s] = rb1.w;
    };
    const int tx = tid & 15, ty = tid >> 4;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    const int KT = K / SG_BK;
    gload(0);
    sstore(0);
    __syncthreads();
    for (int kt = 0; kt < KT; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < KT) gload(kt + 1);
#pragma unroll
        for (int kk = 0; kk < SG_BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][sw_col(kk, ty * 4)]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][sw_col(kk, ty * 4 + 64)]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][sw_col(kk, tx * 4)]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][sw_col(kk, tx * 4 + 64)]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < KT) sstore(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const size_t row = m0 + ty * 4 + (i & 3) + (i >> 2) * 64;
        if (row >= m) continue;
        const float rr1 = r1[row], rr2 = r2[row];
        float *orow = out + row * ldo;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const size_t col = n0 + tx * 4 + (j & 3) + (j >> 2) * 64;
            if (col >= n) continue;
            const float ipt = __fmul_rn(__fmul_rn(acc[i][j], rr1), c1[col]);
            const float d = __fsub_rn(__fadd_rn(rr2, c2[col]), __fmul_rn(2.0f, ipt));
            orow[col] = d > 0.0f ? d : 0.0f;
        }
    }
}

unsigned grid_for(size_t work, int threads) {
    size_t b = (work + threads - 1) / threads;
    const size_t cap = (size_t)148 * 32;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace

cudaError_t launch_planes_from_codes(const Params &P, const DevTables &T, const uint8_t *codes,
                                     size_t rows, size_t rows_pad, bool sym, int fmt, void *plane0,
                                     void *plane1, float *s1, float *s2, cudaStream_t st) {
    if (rows_pad == 0) return cudaSuccess;
    const int K = sym ? P.D : 2 * P.D;
    const int ldl = (!sym && fmt == kPlaneBF16) ? asym_lo_width(P.D) : K;
    planes_from_codes_kernel<<<grid_for(rows_pad * (K / 4), 256), 256, 0, st>>>(
        codes, rows, rows_pad, P, T, sym ? 1 : 0, fmt, ldl, plane0, plane1, s1, s2);
    return cudaGetLastError();
}

cudaError_t launch_dec_factors(const Params &P, const uint8_t *codes, size_t rows, size_t rows_pad,
                               bool sym, float *c1, float *c2, float *fc, float *fs, cudaStream_t st) {
    if (rows_pad == 0) return cudaSuccess;
    const size_t blocks = std::min<size_t>((rows_pad + 255) / 256, 148 * 16);
    dec_factors_kernel<<<(unsigned)blocks, 256, 0, st>>>(codes, rows, rows_pad, P, sym ? 1 : 0, c1, c2,
                                                          fc, fs);
    return cudaGetLastError();
}

cudaError_t launch_planes_from_prepared(const float *q_rot, const float *s_q, const float *norms,
                                        size_t rows, size_t rows_pad, int D, int fmt, void *plane0,
                                        void *plane1, float *r1, float *r2, cudaStream_t st) {
    if (rows_pad == 0) return cudaSuccess;
    planes_from_prepared_kernel<<<grid_for(rows_pad * 2 * D, 256), 256, 0, st>>>(
        q_rot, s_q, norms, rows, rows_pad, D, fmt, plane0, plane1, r1, r2);
    return cudaGetLastError();
}

cudaError_t launch_sgemm_dist(const float *A, const float *B, int K, size_t m, size_t m_pad,
                              size_t n, size_t n_pad, const float *r1, const float *r2,
                              const float *c1, const float *c2, float *out, size_t ldo,
                              cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    if (K % SG_BK || m_pad % SG_BM || n_pad % SG_BN) return cudaErrorInvalidValue;
    if (m_pad / SG_BM > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    // row blocks on grid.x (up to 2^31 - 1), column blocks on grid.y in chunks of 65535
    for (size_t nb = 0; nb < n_pad; nb += (size_t)SG_BN * 65535) {
        const size_t cols = (n_pad - nb < (size_t)SG_BN * 65535) ? (n_pad - nb) : (size_t)SG_BN * 65535;
        dim3 grid((unsigned)(m_pad / SG_BM), (unsigned)(cols / SG_BN));
        sgemm_dist_kernel<<<grid, 256, 0, st>>>(A, B + nb * (size_t)K, K, m, n > nb ? n - nb : 0,
                                               r1, r2, c1 + nb, c2 + nb, out + nb, ldo);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace tq
