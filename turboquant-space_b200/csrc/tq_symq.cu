// tq_symq.cu -- sm_100a kernels of two reference features beside the
// encode-and-scan path:
//
//   rotated_coords_kernel  rotatedCoordsBatch (space_turbo_quant.h:411-435):
//                          the sigma-normalised post-rotation coordinates,
//                          bit-identical to the reference's pinned build.
//   symq_planes_kernel     operand planes of the QJL-corrected symmetric
//                          distances (:483-572, 731-945): per code the
//                          centroid values, the +-1 QJL signs and, for the
//                          full variants, the reconstruction passed through
//                          the QJL Hadamard (randomizedHadamard of c * sigma).
//   symq_gemm_wide_kernel  two FP32 contractions per tile (the MSE term and the
//   / symq_gemm_kernel
//                          correction) with the reference's distance epilogue
//                          fused: corr = clamp(corr, +-|ip_mse|),
//                          ip = (ip_mse + corr) |a| |b|, d = max(0, ...).
//
// The reference evaluates the full variants pair by pair (two
// reconstructions and two Hadamards per pair); here every code is
// reconstructed and rotated once, and the four inner products of a pair
// become one K = D and one K = 3 D contraction:
//   ip_mse = <c_a, c_b> sigma_a sigma_b                (full, light)
//          = <recon_a, recon_b>                        (full prepared)
//   corr   = <[recon_a | s g_a sgn_a | p g_a sgn_a], [s g_b sgn_b | recon_b | g_b sgn_b]>
//          = s g_b <recon_a, sgn_b> + s g_a <sgn_a, recon_b> + p g_a g_b <sgn_a, sgn_b>
//   (s = scale, p = pi / (2 D), g = gamma)             (full, full prepared)
//   corr   = <sgn_a, sgn_b> (p g_a) g_b                (light)
#include "tq_async.cuh"
#include "tq_internal.h"
#include "tq_rht.cuh"

#include <cstdint>

namespace tq {
namespace {

constexpr float kPi = 3.14159265358979323846f;

// ---------------------------------------------------------------------------
// rotatedCoordsBatch: one warp per row.  |x|^2 through the reference's
// reduction tree, inv_norm = 1 / sqrt(|x|^2) (guard 1e-20f), the rotation
// RHT, var over D through the same tree, inv_sigma = sqrt(D / var) (guard
// 1e-20f, else 1), out = rotated * inv_sigma.
// ---------------------------------------------------------------------------
template <int LOG_D>
__global__ void __launch_bounds__(256) rotated_coords_kernel(const float *__restrict__ X, size_t n,
                                                             float *__restrict__ out, Params P,
                                                             DevTables T) {
    constexpr int D = 1 << LOG_D;
    constexpr int VS = D + 8;
    extern __shared__ __align__(16) unsigned char smem[];
    load_tables(smem, P, T, false);
    __syncthreads();
    const uint32_t *s_rot = reinterpret_cast<const uint32_t *>(smem + kTabRotOff);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float *buf = reinterpret_cast<float *>(smem + kTabBytes) + warp * VS;
    for (size_t r = (size_t)blockIdx.x * nw + warp; r < n; r += (size_t)gridDim.x * nw) {
        const float *src = X + r * (size_t)P.dim;
        for (int i = lane; i < D; i += 32) buf[swz(i)] = (i < P.dim) ? src[i] : 0.0f;
        __syncwarp();
        const float ns = chain_sq_reduce(buf, P.dim, lane);
        const float inv_norm = (ns > 1e-20f) ? __fdiv_rn(1.0f, __fsqrt_rn(ns)) : 0.0f;
        __syncwarp();
        fwht_from<LOG_D, 0, true>(buf, lane, inv_norm, s_rot, P.wht_scale);
        const float var = chain_sq_reduce(buf, D, lane);
        const float inv_sigma = (var > 1e-20f) ? __fsqrt_rn(__fdiv_rn((float)D, var)) : 1.0f;
        float *dst = out + r * (size_t)D;
        for (int i = lane; i < D; i += 32) dst[i] = __fmul_rn(buf[swz(i)], inv_sigma);
        __syncwarp();
    }
}

// x rounded to TF32 (10 fraction bits), nearest-even, kept in an FP32
// container with the low 13 bits clear (finite x).
__device__ __forceinline__ float round_tf32(float x) {
    const uint32_t b = __float_as_uint(x);
    return __uint_as_float((b + 0xFFFu + ((b >> 13) & 1u)) & ~0x1FFFu);
}

// ---------------------------------------------------------------------------
// Operand planes: one warp per code.  P1 (ldk1 columns), P2 (ldk2 columns)
// and 8 scalars per row: [s1, norm, s2, gamma, sigma, scale * gamma,
// (pi / 2D) * gamma, 0].  The GEMM uses s1, norm and s2:
//   ip_mse = C1 s1_a s1_b, corr = clamp(C2 s2_a s2_b, +-|ip_mse|).
// Columns past K are written as zeros.
// TF32: each value v is written as the pair hi = tf32(v) (P1 / P2) and
// lo = tf32(v - hi) (L1 / L2; L2 may be null when the second plane holds
// exact values, the light variant's +-1), and rows [rows, rows_pad) are
// zero rows (no scalars).
// ---------------------------------------------------------------------------
template <int LOG_D, bool TF32>
__global__ void __launch_bounds__(256) symq_planes_kernel(const uint8_t *__restrict__ codes,
                                                          size_t rows, size_t rows_pad, int mode,
                                                          int row_side, float *__restrict__ P1,
                                                          float *__restrict__ L1, int ldk1,
                                                          float *__restrict__ P2,
                                                          float *__restrict__ L2, int ldk2,
                                                          float *__restrict__ scal, Params P,
                                                          DevTables T) {
    constexpr int D = 1 << LOG_D;
    constexpr int VS = D + 8;
    extern __shared__ __align__(16) unsigned char smem[];
    load_tables(smem, P, T, true);
    __syncthreads();
    const float *s_cent = reinterpret_cast<const float *>(smem + kTabCentOff);
    const uint32_t *s_qjl = reinterpret_cast<const uint32_t *>(smem + kTabQjlOff);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float *buf = reinterpret_cast<float *>(smem + kTabBytes) + warp * VS;
    const bool recon = mode != SYMQ_LIGHT;
    const float p2d = __fdiv_rn(kPi, __fmul_rn(2.0f, (float)D));  // (float)M_PI / (2.0f * d)
    for (size_t r = (size_t)blockIdx.x * nw + warp; r < rows_pad; r += (size_t)gridDim.x * nw) {
        float *p1 = P1 + r * (size_t)ldk1;
        float *p2 = P2 + r * (size_t)ldk2;
        float *l1 = TF32 ? L1 + r * (size_t)ldk1 : nullptr;
        float *l2 = (TF32 && L2) ? L2 + r * (size_t)ldk2 : nullptr;
        auto put1 = [&](int i, float v) {
            if constexpr (TF32) {
                const float h = round_tf32(v);
                p1[i] = h;
                l1[i] = round_tf32(__fsub_rn(v, h));
            } else {
                p1[i] = v;
            }
        };
        auto put2 = [&](int i, float v) {
            if constexpr (TF32) {
                const float h = round_tf32(v);
                p2[i] = h;
                if (l2) l2[i] = round_tf32(__fsub_rn(v, h));
            } else {
                p2[i] = v;
            }
        };
        if (r >= rows) {  // TF32 padding row
            for (int i = lane; i < ldk1; i += 32) put1(i, 0.0f);
            for (int i = lane; i < ldk2; i += 32) put2(i, 0.0f);
            continue;
        }
        const uint8_t *c = codes + r * (size_t)P.cs;
        float meta[3];  // the trailer may be unaligned (D = 4 nibble codes: pb = 2)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const uint8_t *t = c + P.pb + 4 * q;
            meta[q] = __uint_as_float((uint32_t)t[0] | ((uint32_t)t[1] << 8) |
                                      ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24));
        }
        const float norm = meta[0], gamma = meta[1], sigma = meta[2];
        const float sg = __fmul_rn(P.scale, gamma);
        const float pg = __fmul_rn(p2d, gamma);
        // pass 1: units -> centroid values and signs
        for (int i = lane; i < D; i += 32) {
            unsigned u;
            if (P.nibble) {
                const unsigned b = c[i >> 1];
                u = (i & 1) ? (b >> 4) : (b & 15u);
            } else {
                u = c[i];
            }
            const float cv = s_cent[u >> 1];
            const float sgn = (u & 1u) ? 1.0f : -1.0f;
            if (recon) buf[swz(i)] = __fmul_rn(cv, sigma);
            if (mode == SYMQ_LIGHT) {
                put1(i, cv);
                put2(i, sgn);
            } else if (mode == SYMQ_FULL) {
                put1(i, cv);
            }
            if (mode == SYMQ_FULL || mode == SYMQ_FULL_PREPARED) {
                if (row_side) {
                    put2(D + i, sgn * sg);
                    put2(2 * D + i, sgn * pg);
                } else {
                    put2(i, sgn * sg);
                    put2(2 * D + i, sgn * gamma);
                }
            } else if (mode == SYMQ_PREPARE) {
                put2(i, sgn);
            }
        }
        // pass 2: recon = RHT_qjl(c * sigma)
        if (recon) {
            __syncwarp();
            fwht_from<LOG_D, 0, false>(buf, lane, 1.0f, s_qjl, P.wht_scale);
            for (int i = lane; i < D; i += 32) {
                const float x = buf[swz(i)];
                if (mode != SYMQ_FULL) put1(i, x);
                if (mode == SYMQ_FULL || mode == SYMQ_FULL_PREPARED) put2((row_side ? 0 : D) + i, x);
            }
            __syncwarp();
        }
        const int k2 = (mode == SYMQ_FULL || mode == SYMQ_FULL_PREPARED) ? 3 * D : D;
        for (int i = D + lane; i < ldk1; i += 32) put1(i, 0.0f);
        for (int i = k2 + lane; i < ldk2; i += 32) put2(i, 0.0f);
        if (lane == 0) {
            float *s = scal + 8 * r;
            s[0] = (mode == SYMQ_LIGHT || mode == SYMQ_FULL) ? sigma : 1.0f;
            s[1] = norm;
            s[2] = (mode == SYMQ_LIGHT) ? (row_side ? pg : gamma) : 1.0f;
            s[3] = gamma;
            s[4] = sigma;
            s[5] = sg;
            s[6] = pg;
            s[7] = 0.0f;
        }
    }
}

// The row side of the 1->N prepared scan from a prepared code (recon_q,
// sign_q, [norm, gamma, sigma, scale * gamma, (pi / 2D) * gamma]).
__global__ void symq_prepared_row_kernel(const float *__restrict__ recon,
                                         const float *__restrict__ sign,
                                         const float *__restrict__ sc, int D,
                                         float *__restrict__ P1, int ldk1,
                                         float *__restrict__ P2, int ldk2,
                                         float *__restrict__ scal) {
    for (int i = threadIdx.x; i < ldk1; i += blockDim.x) P1[i] = (i < D) ? recon[i] : 0.0f;
    for (int i = threadIdx.x; i < ldk2; i += blockDim.x) {
        float v = 0.0f;
        if (i < D) v = recon[i];
        else if (i < 2 * D) v = sign[i - D] * sc[3];
        else if (i < 3 * D) v = sign[i - 2 * D] * sc[4];
        P2[i] = v;
    }
    if (threadIdx.x == 0) {
        scal[0] = 1.0f;
        scal[1] = sc[0];
        scal[2] = 1.0f;
        scal[3] = sc[1];
        scal[4] = sc[2];
        scal[5] = sc[3];
        scal[6] = sc[4];
        scal[7] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Two FP32 contractions per 64 x 64 tile, 4 x 4 outputs per thread, K in
// steps of 16 through shared memory (A and B stored K-major, transposed on
// the way in so the inner loop reads float4 rows); then the fused epilogue.
// ---------------------------------------------------------------------------
constexpr int SQ_BM = 64, SQ_BN = 64, SQ_BK = 16;

__device__ __forceinline__ void sq_load_tile(float (*S)[SQ_BM + 4], const float *__restrict__ Pl,
                                             size_t rows, size_t r0, int ldk, int k0, int tid) {
    const int r = tid >> 2, kk = (tid & 3) * 4;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r0 + r < rows) v = *reinterpret_cast<const float4 *>(Pl + (r0 + r) * (size_t)ldk + k0 + kk);
    S[kk + 0][r] = v.x;
    S[kk + 1][r] = v.y;
    S[kk + 2][r] = v.z;
    S[kk + 3][r] = v.w;
}

__device__ __forceinline__ void sq_accumulate(float (&acc)[4][4], const float *__restrict__ Pa,
                                              const float *__restrict__ Pb, size_t m, size_t n,
                                              size_t r0, size_t c0, int ldk,
                                              float (*As)[SQ_BM + 4], float (*Bs)[SQ_BN + 4],
                                              int tid, int tx, int ty) {
    for (int k0 = 0; k0 < ldk; k0 += SQ_BK) {
        sq_load_tile(As, Pa, m, r0, ldk, k0, tid);
        sq_load_tile(Bs, Pb, n, c0, ldk, k0, tid);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < SQ_BK; ++k) {
            const float4 a = *reinterpret_cast<const float4 *>(&As[k][ty * 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&Bs[k][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) symq_gemm_kernel(
    const float *__restrict__ P1a, const float *__restrict__ P2a, const float *__restrict__ sa,
    size_t m, const float *__restrict__ P1b, const float *__restrict__ P2b,
    const float *__restrict__ sb, size_t n, int ldk1, int ldk2, float *__restrict__ out,
    size_t ldo) {
    __shared__ __align__(16) float As[SQ_BK][SQ_BM + 4];
    __shared__ __align__(16) float Bs[SQ_BK][SQ_BN + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const size_t r0 = (size_t)blockIdx.y * SQ_BM, c0 = (size_t)blockIdx.x * SQ_BN;
    float acc1[4][4] = {}, acc2[4][4] = {};
    sq_accumulate(acc1, P1a, P1b, m, n, r0, c0, ldk1, As, Bs, tid, tx, ty);
    sq_accumulate(acc2, P2a, P2b, m, n, r0, c0, ldk2, As, Bs, tid, tx, ty);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const size_t r = r0 + ty * 4 + i;
        if (r >= m) break;
        const float s1a = sa[8 * r], na = sa[8 * r + 1], s2a = sa[8 * r + 2];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const size_t c = c0 + tx * 4 + j;
            if (c >= n) break;
            const float s1b = sb[8 * c], nb = sb[8 * c + 1], s2b = sb[8 * c + 2];
            const float ip_mse = __fmul_rn(__fmul_rn(acc1[i][j], s1a), s1b);
            const float lim = fabsf(ip_mse);
            float corr = __fmul_rn(__fmul_rn(acc2[i][j], s2a), s2b);
            corr = fmaxf(-lim, fminf(lim, corr));
            const float ip = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), na), nb);
            const float d = __fsub_rn(__fadd_rn(__fmul_rn(na, na), __fmul_rn(nb, nb)),
                                      __fmul_rn(2.0f, ip));
            out[r * ldo + c] = d > 0.0f ? d : 0.0f;
        }
    }
}

// ---------------------------------------------------------------------------
// The same two contractions with 128 x 128 tiles and 8 x 8 outputs per thread
// (half the shared-memory reads per FMA of the 64 x 64 kernel, which is bound
// by them): C1 is accumulated first and parked in shared memory (64 floats
// per thread, 64 KB), then C2 in the same registers; the epilogue combines
// them as above.  K step 16, double-buffered transposed tiles whose columns
// are XOR-swizzled with bit 3 of k (conflict-free stores); rows past m or n
// load as zeros.  128 registers, two CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int SQW_BM = 128, SQW_BK = 16, SQW_PAD = 4;
constexpr size_t kSqwStashBytes = (size_t)64 * 256 * 4;

__device__ __forceinline__ int sqw_col(int k, int col) { return col ^ (((k >> 3) & 1) << 3); }

__device__ __forceinline__ void sqw_accumulate(float (&acc)[8][8], const float *__restrict__ Pa,
                                               const float *__restrict__ Pb, size_t m, size_t n,
                                               size_t r0, size_t c0, int ldk,
                                               float (*As)[SQW_BK][SQW_BM + SQW_PAD],
                                               float (*Bs)[SQW_BK][SQW_BM + SQW_PAD], int tid) {
    const int lrow = tid >> 2, lk = (tid & 3) * 4, tx = tid & 15, ty = tid >> 4;
    const bool a0ok = r0 + lrow < m, a1ok = r0 + lrow + 64 < m;
    const bool b0ok = c0 + lrow < n, b1ok = c0 + lrow + 64 < n;
    const float *Ag0 = Pa + (a0ok ? (r0 + lrow) * (size_t)ldk : 0) + lk;
    const float *Ag1 = Pa + (a1ok ? (r0 + lrow + 64) * (size_t)ldk : 0) + lk;
    const float *Bg0 = Pb + (b0ok ? (c0 + lrow) * (size_t)ldk : 0) + lk;
    const float *Bg1 = Pb + (b1ok ? (c0 + lrow + 64) * (size_t)ldk : 0) + lk;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 ra0, ra1, rb0, rb1;
    auto gload = [&](int kt) {
        const size_t o = (size_t)kt * SQW_BK;
        ra0 = a0ok ? __ldg(reinterpret_cast<const float4 *>(Ag0 + o)) : z;
        ra1 = a1ok ? __ldg(reinterpret_cast<const float4 *>(Ag1 + o)) : z;
        rb0 = b0ok ? __ldg(reinterpret_cast<const float4 *>(Bg0 + o)) : z;
        rb1 = b1ok ? __ldg(reinterpret_cast<const float4 *>(Bg1 + o)) : z;
    };
    const int s0 = sqw_col(lk, lrow), s1 = sqw_col(lk, lrow + 64);
    auto sstore = [&](int buf) {
        As[buf][lk + 0][s0] = ra0.x; As[buf][lk + 1][s0] = ra0.y;
        As[buf][lk + 2][s0] = ra0.z; As[buf][lk + 3][s0] = ra0.w;
        As[buf][lk + 0][s1] = ra1.x; As[buf][lk + 1][s1] = ra1.y;
        As[buf][lk + 2][s1] = ra1.z; As[buf][lk + 3][s1] = ra1.w;
        Bs[buf][lk + 0][s0] = rb0.x; Bs[buf][lk + 1][s0] = rb0.y;
        Bs[buf][lk + 2][s0] = rb0.z; Bs[buf][lk + 3][s0] = rb0.w;
        Bs[buf][lk + 0][s1] = rb1.x; Bs[buf][lk + 1][s1] = rb1.y;
        Bs[buf][lk + 2][s1] = rb1.z; Bs[buf][lk + 3][s1] = rb1.w;
    };
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    const int KT = ldk / SQW_BK;
    gload(0);
    sstore(0);
    __syncthreads();
    for (int kt = 0; kt < KT; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < KT) gload(kt + 1);
#pragma unroll
        for (int kk = 0; kk < SQW_BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][sqw_col(kk, ty * 4)]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][sqw_col(kk, ty * 4 + 64)]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][sqw_col(kk, tx * 4)]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][sqw_col(kk, tx * 4 + 64)]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < KT) sstore(buf ^ 1);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256, 2) symq_gemm_wide_kernel(
    const float *__restrict__ P1a, const float *__restrict__ P2a, const float *__restrict__ sa,
    size_t m, const float *__restrict__ P1b, const float *__restrict__ P2b,
    const float *__restrict__ sb, size_t n, int ldk1, int ldk2, float *__restrict__ out,
    size_t ldo) {
    __shared__ __align__(16) float As[2][SQW_BK][SQW_BM + SQW_PAD];
    __shared__ __align__(16) float Bs[2][SQW_BK][SQW_BM + SQW_PAD];
    extern __shared__ float stash[];  // [64][256]: value i * 8 + j of thread tid at [(i * 8 + j) * 256 + tid]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    // row blocks on grid.x (fastest): CTAs running together share the column tile in L2
    const size_t r0 = (size_t)blockIdx.x * SQW_BM, c0 = (size_t)blockIdx.y * SQW_BM;
    float acc[8][8];
    sqw_accumulate(acc, P1a, P1b, m, n, r0, c0, ldk1, As, Bs, tid);
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) stash[(i * 8 + j) * 256 + tid] = acc[i][j];
    sqw_accumulate(acc, P2a, P2b, m, n, r0, c0, ldk2, As, Bs, tid);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const size_t r = r0 + ty * 4 + (i & 3) + (i >> 2) * 64;
        if (r >= m) continue;
        const float s1a = sa[8 * r], na = sa[8 * r + 1], s2a = sa[8 * r + 2];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const size_t c = c0 + tx * 4 + (j & 3) + (j >> 2) * 64;
            if (c >= n) continue;
            const float s1b = sb[8 * c], nb = sb[8 * c + 1], s2b = sb[8 * c + 2];
            const float ip_mse = __fmul_rn(__fmul_rn(stash[(i * 8 + j) * 256 + tid], s1a), s1b);
            const float lim = fabsf(ip_mse);
            float corr = __fmul_rn(__fmul_rn(acc[i][j], s2a), s2b);
            corr = fmaxf(-lim, fminf(lim, corr));
            const float ip = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), na), nb);
            const float d = __fsub_rn(__fadd_rn(__fmul_rn(na, na), __fmul_rn(nb, nb)),
                                      __fmul_rn(2.0f, ip));
            out[r * ldo + c] = d > 0.0f ? d : 0.0f;
        }
    }
}

template <template <int> class F, typename... Args>
cudaError_t dispatch_logd_sq(int log2D, Args &&...args) {
    switch (log2D) {
        case 2: return F<2>::run(args...);
        case 3: return F<3>::run(args...);
        case 4: return F<4>::run(args...);
        case 5: return F<5>::run(args...);
        case 6: return F<6>::run(args...);
        case 7: return F<7>::run(args...);
        case 8: return F<8>::run(args...);
        case 9: return F<9>::run(args...);
        case 10: return F<10>::run(args...);
        case 11: return F<11>::run(args...);
        case 12: return F<12>::run(args...);
        case 13: return F<13>::run(args...);
        default: return cudaErrorInvalidValue;
    }
}

int sq_sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 148;
    }
    return count;
}

// warps per block for one D-float buffer per warp (at most 8, 200 KB)
int sq_warps(int D) {
    int w = (200 * 1024 - kTabBytes) / (4 * (D + 8));
    return w > 8 ? 8 : (w < 1 ? 1 : w);
}

template <int LOG_D>
struct RotRun {
    static cudaError_t run(const Params &P, const DevTables &T, const float *X, size_t n,
                           float *out, cudaStream_t st) {
        const int D = 1 << LOG_D, w = sq_warps(D);
        const size_t smem = (size_t)kTabBytes + (size_t)w * 4 * (D + 8);
        cudaError_t e = cudaFuncSetAttribute(rotated_coords_kernel<LOG_D>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        size_t blocks = (n + w - 1) / w;
        const size_t cap = (size_t)sq_sm_count() * 8;
        if (blocks > cap) blocks = cap;
        rotated_coords_kernel<LOG_D><<<(unsigned)blocks, 32 * w, smem, st>>>(X, n, out, P, T);
        return cudaGetLastError();
    }
};

template <int LOG_D>
struct PlanesRun {
    template <bool TF32>
    static cudaError_t go(const Params &P, const DevTables &T, const uint8_t *codes, size_t rows,
                          size_t rows_pad, int mode, int row_side, float *P1, float *L1, int ldk1,
                          float *P2, float *L2, int ldk2, float *scal, cudaStream_t st) {
        const int D = 1 << LOG_D, w = sq_warps(D);
        const size_t smem = (size_t)kTabBytes + (size_t)w * 4 * (D + 8);
        cudaError_t e = cudaFuncSetAttribute(symq_planes_kernel<LOG_D, TF32>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        size_t blocks = (rows_pad + w - 1) / w;
        const size_t cap = (size_t)sq_sm_count() * 8;
        if (blocks > cap) blocks = cap;
        symq_planes_kernel<LOG_D, TF32><<<(unsigned)blocks, 32 * w, smem, st>>>(
            codes, rows, rows_pad, mode, row_side, P1, L1, ldk1, P2, L2, ldk2, scal, P, T);
        return cudaGetLastError();
    }
    static cudaError_t run(const Params &P, const DevTables &T, const uint8_t *codes, size_t rows,
                           size_t rows_pad, int mode, int row_side, float *P1, float *L1, int ldk1,
                           float *P2, float *L2, int ldk2, float *scal, cudaStream_t st) {
        if (L1) return go<true>(P, T, codes, rows, rows_pad, mode, row_side, P1, L1, ldk1, P2, L2, ldk2,
                                scal, st);
        return go<false>(P, T, codes, rows, rows, mode, row_side, P1, nullptr, ldk1, P2, nullptr, ldk2,
                         scal, st);
    }
};

}  // namespace

int symq_ldk(int K) { return (K + SQ_BK - 1) / SQ_BK * SQ_BK; }

int symq_k2(int mode, int D) {
    return (mode == SYMQ_FULL || mode == SYMQ_FULL_PREPARED) ? 3 * D : D;
}

cudaError_t launch_rotated_coords(const Params &P, const DevTables &T, const float *X, size_t n,
                                  float *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    return dispatch_logd_sq<RotRun>(P.log2D, P, T, X, n, out, st);
}

cudaError_t launch_symq_planes(const Params &P, const DevTables &T, const uint8_t *codes,
                               size_t rows, int mode, bool row_side, float *P1, int ldk1,
                               float *P2, int ldk2, float *scal, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    return dispatch_logd_sq<PlanesRun>(P.log2D, P, T, codes, rows, rows, mode, (int)row_side, P1,
                                       (float *)nullptr, ldk1, P2, (float *)nullptr, ldk2, scal, st);
}

cudaError_t launch_symq_planes_tf32(const Params &P, const DevTables &T, const uint8_t *codes,
                                    size_t rows, size_t rows_pad, int mode, bool row_side,
                                    float *H1, float *L1, int K1, float *H2, float *L2, int K2,
                                    float *scal, cudaStream_t st) {
    if (rows_pad == 0) return cudaSuccess;
    if (!H1 || !L1 || !H2 || rows > rows_pad || K1 < (1 << P.log2D) ||
        K2 < symq_k2(mode, 1 << P.log2D))
        return cudaErrorInvalidValue;
    return dispatch_logd_sq<PlanesRun>(P.log2D, P, T, codes, rows, rows_pad, mode, (int)row_side, H1,
                                       L1, K1, H2, L2, K2, scal, st);
}

cudaError_t launch_symq_prepared_row(const float *recon, const float *sign, const float *sc, int D,
                                     float *P1, int ldk1, float *P2, int ldk2, float *scal,
                                     cudaStream_t st) {
    symq_prepared_row_kernel<<<1, 256, 0, st>>>(recon, sign, sc, D, P1, ldk1, P2, ldk2, scal);
    return cudaGetLastError();
}

cudaError_t launch_symq_gemm(const float *P1a, const float *P2a, const float *sa, size_t m,
                             const float *P1b, const float *P2b, const float *sb, size_t n,
                             int ldk1, int ldk2, float *out, size_t ldo, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    if (ldk1 % SQW_BK || ldk2 % SQW_BK) return cudaErrorInvalidValue;
    if (m >= 64) {
        // 128 x 128 tiles: row blocks on grid.x, column blocks on grid.y in chunks of 65535
        cudaError_t e = cudaFuncSetAttribute(symq_gemm_wide_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSqwStashBytes);
        if (e != cudaSuccess) return e;
        const size_t gx = (m + SQW_BM - 1) / SQW_BM;
        if (gx > 0x7FFFFFFFull) return cudaErrorInvalidValue;
        const size_t nblk = (n + SQW_BM - 1) / SQW_BM;
        for (size_t y0 = 0; y0 < nblk; y0 += 65535) {
            const size_t gy = (nblk - y0 < 65535) ? nblk - y0 : 65535;
            const size_t cc = y0 * SQW_BM;
            symq_gemm_wide_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, kSqwStashBytes, st>>>(
                P1a, P2a, sa, m, P1b + cc * (size_t)ldk1, P2b + cc * (size_t)ldk2, sb + 8 * cc,
                n - cc, ldk1, ldk2, out + cc, ldo);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const size_t gx = (n + SQ_BN - 1) / SQ_BN;
    for (size_t y0 = 0; y0 < (m + SQ_BM - 1) / SQ_BM; y0 += 65535) {
        const size_t gy = ((m + SQ_BM - 1) / SQ_BM - y0 < 65535) ? (m + SQ_BM - 1) / SQ_BM - y0 : 65535;
        const size_t rr = y0 * SQ_BM;
        symq_gemm_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, 0, st>>>(
            P1a + rr * (size_t)ldk1, P2a + rr * (size_t)ldk2, sa + 8 * rr, m - rr, P1b, P2b, sb, n,
            ldk1, ldk2, out + rr * ldo, ldo);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace tq
