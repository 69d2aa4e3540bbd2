// tq_tc.cu -- split-BF16 tensor-core contraction of the M x N distances on
// sm_100a (tcgen05 + TMA), with the distance epilogue fused.
//
// C = Ah Bh^T + Ah Bl^T + Al Bh^T over BF16 hi/lo operand planes (x = hi + lo,
// see tq_mton.cu), accumulated in FP32 in tensor memory; then
// d = max(0, r2_i + c2_j - 2 (C_ij r1_i) c1_j) is written to out.  K blocks
// from kbx on have an exact B (lo = 0: the +-1 QJL half of asymmetric planes):
// there the Bl tile is not loaded and Ah Bl^T is not issued.
//
// Persistent kernel, one CTA per SM, 6 warps:
//   warp 0      TMA producer: per K block of 64, loads Ah, Al (128 x 64) and
//               Bh, Bl (256 x 64; Bl only below kbx) tiles, 128-byte
//               swizzled, into a 2-stage ring
//   warp 1      allocates 512 TMEM columns (two 128 x 256 FP32 accumulators);
//               one thread issues 3 tcgen05.mma (M128 N256 K16) per K step
//               (2 from kbx on)
//               and commits to the stage's "empty" barrier and, after a
//               tile's last K block, to the accumulator's "full" barrier
//   warps 2..5  epilogue: tcgen05.ld 32x32b rows of the accumulator, apply the
//               distance formula, store; then release the accumulator
// Tiles are visited with the A-block index fastest so that CTAs running at the
// same time share the B tile in L2.  Every mbarrier wait is bounded: after
// ~2 s it records an error code in *err and the CTA winds down (frees its
// tensor memory) instead of waiting forever.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "tq_async.cuh"
#include "tq_mton.h"

namespace tq {
namespace {

constexpr int TC_BM = 128, TC_BN = 256, TC_BK = 64, TC_STAGES = 2;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;   // 16 KB
constexpr int TC_B_BYTES = TC_BN * TC_BK * 2;   // 32 KB
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;  // 96 KB
constexpr int TC_TMEM_COLS = 512;
constexpr int TC_THREADS = 192;
// error codes written to *err
constexpr int kErrFull = 1, kErrEmpty = 2, kErrTmemFull = 3, kErrTmemEmpty = 4;

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile whose
// rows are 128 bytes (64 BF16) and whose 8-row groups are 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);  // start address
    d |= (uint64_t)1u << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;        // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                  // layout: SWIZZLE_128B
    return d;
}

// Instruction descriptor: kind::f16, BF16 x BF16 -> FP32, both K-major, M128 N256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                            ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_i(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(TC_THREADS, 1) tc_dist_kernel(
    const __grid_constant__ CUtensorMap tm_ah, const __grid_constant__ CUtensorMap tm_al,
    const __grid_constant__ CUtensorMap tm_bh, const __grid_constant__ CUtensorMap tm_bl, int K,
    int kbx, unsigned num_mb, unsigned num_tiles, size_t m, size_t n, const float *__restrict__ r1,
    const float *__restrict__ r2, const float *__restrict__ c1, const float *__restrict__ c2,
    float *__restrict__ out, size_t ldo, int *err) {
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TC_STAGES * TC_STAGE_BYTES);
    // bars: full[2], empty[2], tfull[2], tempty[2], drain; then the TMEM address slot
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 9);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + 2);
    const uint32_t tfull0 = smem_u32(bars + 4), tempty0 = smem_u32(bars + 6);
    const uint32_t drain = smem_u32(bars + 8);

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull0 + 8 * b, 1);
            mbar_init(tempty0 + 8 * b, 128);
        }
        mbar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int KB = K / TC_BK;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (unsigned tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
                const int mb = (int)(tile % num_mb), nb = (int)(tile / num_mb);
                for (int kb = 0; kb < KB; ++kb, ++it) {
                    const uint32_t s = it % TC_STAGES, ph = (it / TC_STAGES) & 1u;
                    if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err, kErrEmpty)) { ok = false; break; }
                    const uint32_t base = smem_u32(smem + s * TC_STAGE_BYTES);
                    const uint32_t fb = full0 + 8 * s;
                    const bool lo = kb < kbx;
                    mbar_expect_tx(fb, lo ? TC_STAGE_BYTES : TC_STAGE_BYTES - TC_B_BYTES);
                    tma_load_2d(base, &tm_ah, kb * TC_BK, mb * TC_BM, fb);
                    tma_load_2d(base + TC_A_BYTES, &tm_al, kb * TC_BK, mb * TC_BM, fb);
                    tma_load_2d(base + 2 * TC_A_BYTES, &tm_bh, kb * TC_BK, nb * TC_BN, fb);
                    if (lo)
                        tma_load_2d(base + 2 * TC_A_BYTES + TC_B_BYTES, &tm_bl, kb * TC_BK,
                                    nb * TC_BN, fb);
                }
            }
            // drain: every stage issued must have landed before the CTA exits
            for (uint32_t k = 0; k < TC_STAGES && k < it; ++k) {
                const uint32_t j = it - 1 - k;
                mbar_wait(full0 + 8 * (j % TC_STAGES), (j / TC_STAGES) & 1u, err, kErrFull);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t it = 0, t = 0;
            bool ok = true;
            for (unsigned tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x, ++t) {
                const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
                if (!mbar_wait(tempty0 + 8 * b, tph ^ 1u, err, kErrTmemEmpty)) { ok = false; break; }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + b * TC_BN;
                for (int kb = 0; kb < KB; ++kb, ++it) {
                    const uint32_t s = it % TC_STAGES, ph = (it / TC_STAGES) & 1u;
                    if (!mbar_wait(full0 + 8 * s, ph, err, kErrFull)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t base = smem_u32(smem + s * TC_STAGE_BYTES);
                    const uint32_t ah = base, al = base + TC_A_BYTES;
                    const uint32_t bh = base + 2 * TC_A_BYTES, bl = bh + TC_B_BYTES;
                    const bool lo = kb < kbx;
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 16; ++kk) {
                        const uint32_t koff = kk * 32;  // 16 BF16 along K
                        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                        umma(d_tmem, sw128_desc(ah + koff), sw128_desc(bh + koff), acc);
                        if (lo) umma(d_tmem, sw128_desc(ah + koff), sw128_desc(bl + koff), 1u);
                        umma(d_tmem, sw128_desc(al + koff), sw128_desc(bh + koff), 1u);
                    }
                    umma_commit(empty0 + 8 * s);  // smem stage free once these MMAs are done
                }
                if (ok) umma_commit(tfull0 + 8 * b);  // accumulator ready
            }
            // every MMA issued must be complete before the tensor memory is freed
            umma_commit(drain);
            mbar_wait(drain, 0, err, kErrFull);
        }
    } else {
        // ---------------- epilogue (warps 2..5, 128 threads) ----------------
        const int q = warp & 3;           // TMEM lane quadrant this warp may access
        const int row_in_tile = 32 * q + lane;
        uint32_t t = 0;
        for (unsigned tile = blockIdx.x; tile < num_tiles; tile += gridDim.x, ++t) {
            const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
            if (!mbar_wait(tfull0 + 8 * b, tph, err, kErrTmemFull)) break;
            tc_fence_after();
            const int mb = (int)(tile % num_mb), nb = (int)(tile / num_mb);
            const size_t row = (size_t)mb * TC_BM + row_in_tile;
            const bool row_ok = row < m;
            const float rr1 = row_ok ? __ldg(r1 + row) : 0.0f;
            const float rr2 = row_ok ? __ldg(r2 + row) : 0.0f;
            float *orow = out + row * ldo;
            const bool vec = ((ldo & 3) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
#pragma unroll 1
            for (int ch = 0; ch < TC_BN / 32; ++ch) {
                uint32_t r[32];
                __syncwarp();
                tmem_ld32(tmem_base + ((uint32_t)(32 * q) << 16) + b * TC_BN + ch * 32, r);
                const size_t col0 = (size_t)nb * TC_BN + ch * 32;
                if (row_ok && col0 < n) {
                float dv[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const size_t col = col0 + j;
                    const float cc1 = (col < n) ? __ldg(c1 + col) : 0.0f;
                    const float cc2 = (col < n) ? __ldg(c2 + col) : 0.0f;
                    const float ipt = __fmul_rn(__fmul_rn(__uint_as_float(r[j]), rr1), cc1);
                    const float d = __fsub_rn(__fadd_rn(rr2, cc2), __fmul_rn(2.0f, ipt));
                    dv[j] = d > 0.0f ? d : 0.0f;
                }
                if (vec && col0 + 32 <= n) {
                    float4 *o4 = reinterpret_cast<float4 *>(orow + col0);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        o4[j] = make_float4(dv[4 * j], dv[4 * j + 1], dv[4 * j + 2], dv[4 * j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (col0 + j < n) orow[col0 + j] = dv[j];
                }
                }
            }
            __syncwarp();
            tc_fence_before();
            mbar_arrive(tempty0 + 8 * b);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// tc_topk_kernel: the same contraction over a device-resident index, with the
// distances reduced to a per-row top-k instead of being stored.  The number of
// query rows m is read from device memory (so that one captured launch serves
// batches of any size up to the buffers' capacity).  CTA c takes row block
// c / S and the contiguous slice c % S of the column tiles, S = grid / row
// blocks; each epilogue thread keeps its row's best k (distance, index) pairs,
// ties broken by the smaller index, and writes them to the partial buffers
// part_d / part_i [(block * S + slice) * 128 + row][kTopKMax].
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool better(float d, int i, float bd, int bi) {
    return d < bd || (d == bd && i < bi);
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_topk_kernel(
    const __grid_constant__ CUtensorMap tm_ah, const __grid_constant__ CUtensorMap tm_al,
    const __grid_constant__ CUtensorMap tm_bh, const __grid_constant__ CUtensorMap tm_bl, int K,
    int kbx, const int *__restrict__ m_dev, unsigned nb_tiles, size_t n, const float *__restrict__ r1,
    const float *__restrict__ r2, const float *__restrict__ c1, const float *__restrict__ c2, int k,
    float *__restrict__ part_d, int *__restrict__ part_i, int *err) {
    constexpr int B_BYTES = BN * TC_BK * 2;
    constexpr int STAGE_BYTES = 2 * TC_A_BYTES + 2 * B_BYTES;
    constexpr int TMEM_COLS = 2 * BN;
    constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(TC_BM >> 4) << 24);
    const int m = *m_dev;
    const int num_mb = (m + TC_BM - 1) / TC_BM;
    if (num_mb <= 0 || num_mb > (int)gridDim.x) return;
    const int S = (int)gridDim.x / num_mb;
    if ((int)blockIdx.x >= num_mb * S) return;  // uniform over the CTA
    const int mb = (int)blockIdx.x / S, slice = (int)blockIdx.x % S;
    const unsigned nb0 = (unsigned)(((size_t)nb_tiles * slice) / S);
    const unsigned nb1 = (unsigned)(((size_t)nb_tiles * (slice + 1)) / S);
    const unsigned ntiles = nb1 - nb0;

    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], tfull[2], tempty[2], drain; then the TMEM slot
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 5);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
    const uint32_t tfull0 = smem_u32(bars + 2 * STAGES), tempty0 = smem_u32(bars + 2 * STAGES + 2);
    const uint32_t drain = smem_u32(bars + 2 * STAGES + 4);
    if (threadIdx.x == 0) {
        for (int st = 0; st < STAGES; ++st) {
            mbar_init(full0 + 8 * st, 1);
            mbar_init(empty0 + 8 * st, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull0 + 8 * b, 1);
            mbar_init(tempty0 + 8 * b, 128);
        }
        mbar_init(drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int KB = K / TC_BK;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (unsigned t = 0; t < ntiles && ok; ++t) {
                const int nb = (int)(nb0 + t);
                for (int kb = 0; kb < KB; ++kb, ++it) {
                    const uint32_t st = it % STAGES, ph = (it / STAGES) & 1u;
                    if (!mbar_wait(empty0 + 8 * st, ph ^ 1u, err, kErrEmpty)) { ok = false; break; }
                    const uint32_t base = smem_u32(smem + st * STAGE_BYTES);
                    const uint32_t fb = full0 + 8 * st;
                    const bool lo = kb < kbx;
                    mbar_expect_tx(fb, lo ? STAGE_BYTES : STAGE_BYTES - B_BYTES);
                    tma_load_2d(base, &tm_ah, kb * TC_BK, mb * TC_BM, fb);
                    tma_load_2d(base + TC_A_BYTES, &tm_al, kb * TC_BK, mb * TC_BM, fb);
                    tma_load_2d(base + 2 * TC_A_BYTES, &tm_bh, kb * TC_BK, nb * BN, fb);
                    if (lo)
                        tma_load_2d(base + 2 * TC_A_BYTES + B_BYTES, &tm_bl, kb * TC_BK, nb * BN,
                                    fb);
                }
            }
            const uint32_t drain_n = it < (uint32_t)STAGES ? it : (uint32_t)STAGES;
            for (uint32_t q = 0; q < drain_n; ++q) {
                const uint32_t j = it - 1 - q;
                mbar_wait(full0 + 8 * (j % STAGES), (j / STAGES) & 1u, err, kErrFull);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (unsigned t = 0; t < ntiles && ok; ++t) {
                const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
                if (!mbar_wait(tempty0 + 8 * b, tph ^ 1u, err, kErrTmemEmpty)) { ok = false; break; }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + b * BN;
                for (int kb = 0; kb < KB; ++kb, ++it) {
                    const uint32_t st = it % STAGES, ph = (it / STAGES) & 1u;
                    if (!mbar_wait(full0 + 8 * st, ph, err, kErrFull)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t base = smem_u32(smem + st * STAGE_BYTES);
                    const uint32_t ah = base, al = base + TC_A_BYTES;
                    const uint32_t bh = base + 2 * TC_A_BYTES, bl = bh + B_BYTES;
                    const bool lo = kb < kbx;
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 16; ++kk) {
                        const uint32_t koff = kk * 32;
                        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                        umma_i(d_tmem, sw128_desc(ah + koff), sw128_desc(bh + koff), IDESC, acc);
                        if (lo)
                            umma_i(d_tmem, sw128_desc(ah + koff), sw128_desc(bl + koff), IDESC, 1u);
                        umma_i(d_tmem, sw128_desc(al + koff), sw128_desc(bh + koff), IDESC, 1u);
                    }
                    umma_commit(empty0 + 8 * st);
                }
                if (ok) umma_commit(tfull0 + 8 * b);
            }
            umma_commit(drain);
            mbar_wait(drain, 0, err, kErrFull);
        }
    } else {
        const int q = warp & 3;
        const int row_in_tile = 32 * q + lane;
        const int row = mb * TC_BM + row_in_tile;
        const bool row_ok = row < m;
        const float rr1 = row_ok ? __ldg(r1 + row) : 0.0f;
        const float rr2 = row_ok ? __ldg(r2 + row) : 0.0f;
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int t = 0; t < kTopKMax; ++t) {
            bd[t] = INFINITY;
            bi[t] = 0x7fffffff;
        }
        float thr_d = INFINITY;
        int thr_i = 0x7fffffff;
        for (unsigned t = 0; t < ntiles; ++t) {
            const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
            if (!mbar_wait(tfull0 + 8 * b, tph, err, kErrTmemFull)) break;
            tc_fence_after();
            const size_t colbase = (size_t)(nb0 + t) * BN;
#pragma unroll 1
            for (int ch = 0; ch < BN / 32; ++ch) {
                uint32_t r[32];
                __syncwarp();
                tmem_ld32(tmem_base + ((uint32_t)(32 * q) << 16) + b * BN + ch * 32, r);
                const size_t col0 = colbase + ch * 32;
                if (row_ok) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const size_t col = col0 + j;
                        if (col >= n) break;
                        const float ipt = __fmul_rn(__fmul_rn(__uint_as_float(r[j]), rr1), __ldg(c1 + col));
                        float d = __fsub_rn(__fadd_rn(rr2, __ldg(c2 + col)), __fmul_rn(2.0f, ipt));
                        d = d > 0.0f ? d : 0.0f;
                        const int ci = (int)col;
                        if (better(d, ci, thr_d, thr_i)) {
                            float cd = d;
                            int cx = ci;
#pragma unroll
                            for (int u = 0; u < kTopKMax; ++u) {
                                if (u < k) {
                                    const bool sw = better(cd, cx, bd[u], bi[u]);
                                    const float td = bd[u];
                                    const int ti = bi[u];
                                    bd[u] = sw ? cd : td;
                                    bi[u] = sw ? cx : ti;
                                    cd = sw ? td : cd;
                                    cx = sw ? ti : cx;
                                }
                            }
#pragma unroll
                            for (int u = 0; u < kTopKMax; ++u)
                                if (u == k - 1) {
                                    thr_d = bd[u];
                                    thr_i = bi[u];
                                }
                        }
                    }
                }
            }
            __syncwarp();
            tc_fence_before();
            mbar_arrive(tempty0 + 8 * b);
        }
        if (row_ok) {
            const size_t o = ((size_t)blockIdx.x * TC_BM + row_in_tile) * kTopKMax;
#pragma unroll
            for (int u = 0; u < kTopKMax; ++u)
                if (u < k) {
                    part_d[o + u] = bd[u];
                    part_i[o + u] = bi[u];
                }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

// Merge of the per-slice candidates: one warp per query row.  Each lane keeps
// the best k of its slices, then k rounds of a warp arg-min on (d, index)
// produce the sorted top-k.
__global__ void __launch_bounds__(256) topk_merge_kernel(const int *__restrict__ m_dev, int slices_cap,
                                                         int grid_ctas, const float *__restrict__ part_d,
                                                         const int *__restrict__ part_i, int k,
                                                         float *__restrict__ out_d,
                                                         long long *__restrict__ out_i) {
    const int m = *m_dev;
    const int num_mb = (m + TC_BM - 1) / TC_BM;
    if (num_mb <= 0 || num_mb > grid_ctas) return;
    const int S = grid_ctas / num_mb;
    (void)slices_cap;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < m; row += gridDim.x * wpb) {
        const int mb = row / TC_BM, rit = row % TC_BM;
        float bd[kTopKMax];
        int bi[kTopKMax];
#pragma unroll
        for (int t = 0; t < kTopKMax; ++t) {
            bd[t] = INFINITY;
            bi[t] = 0x7fffffff;
        }
        for (int sl = lane; sl < S; sl += 32) {
            const size_t o = ((size_t)(mb * S + sl) * TC_BM + rit) * kTopKMax;
            for (int u = 0; u < k; ++u) {
                float cd = part_d[o + u];
                int cx = part_i[o + u];
#pragma unroll
                for (int v = 0; v < kTopKMax; ++v) {
                    if (v < k) {
                        const bool sw = better(cd, cx, bd[v], bi[v]);
                        const float td = bd[v];
                        const int ti = bi[v];
                        bd[v] = sw ? cd : td;
                        bi[v] = sw ? cx : ti;
                        cd = sw ? td : cd;
                        cx = sw ? ti : cx;
                    }
                }
            }
        }
        // k rounds: warp arg-min of each lane's current head
        int head = 0;
        for (int u = 0; u < k; ++u) {
            float hd = INFINITY;
            int hx = 0x7fffffff;
#pragma unroll
            for (int v = 0; v < kTopKMax; ++v)
                if (v == head) {
                    hd = bd[v];
                    hx = bi[v];
                }
            float wd = hd;
            int wx = hx;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float od = __shfl_xor_sync(0xffffffffu, wd, off);
                const int ox = __shfl_xor_sync(0xffffffffu, wx, off);
                if (better(od, ox, wd, wx)) {
                    wd = od;
                    wx = ox;
                }
            }
            if (hx == wx && hd == wd && head < k) ++head;  // the winning lane pops its head
            if (lane == 0) {
                out_d[(size_t)row * k + u] = wd;
                out_i[(size_t)row * k + u] = (wx == 0x7fffffff) ? -1 : (long long)wx;
            }
        }
    }
}

// Self-test of the bounded wait: one thread waits on an mbarrier that nothing
// arrives at, with a budget of `budget_cycles`; the wait must give up and
// record kErrSelfTest in *err instead of hanging.
constexpr int kErrSelfTest = 9;
__global__ void bounded_wait_selftest_kernel(int *err, long long budget_cycles) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    const uint32_t b = smem_u32(&bar);
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const long long t0 = clock64();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(b, 0)) return;  // cannot happen: no arrival
        if ((it & 255u) == 0 && clock64() - t0 > budget_cycles) {
            atomicCAS(err, 0, kErrSelfTest);
            return;
        }
    }
}

// ---- host: tensor maps ------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool make_map(CUtensorMap *map, const void *base, int K, size_t rows, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int STAGES>
cudaError_t topk_variant(const void *Ah, const void *Al, size_t rows_pad, const void *Bh,
                         const void *Bl, size_t n_pad, int K, int k_lo, const int *m_dev, size_t n,
                         const float *r1, const float *r2, const float *c1, const float *c2, int k,
                         float *part_d, int *part_i, int *err, int grid, cudaStream_t st) {
    if (K % TC_BK || k_lo % TC_BK || k_lo <= 0 || k_lo > K || rows_pad % TC_BM || n_pad % BN)
        return cudaErrorInvalidValue;
    for (const void *p : {Ah, Al, Bh, Bl})
        if (reinterpret_cast<uintptr_t>(p) & 15) return cudaErrorMisalignedAddress;
    alignas(64) CUtensorMap mah, mal, mbh, mbl;
    if (!make_map(&mah, Ah, K, rows_pad, TC_BM) || !make_map(&mal, Al, K, rows_pad, TC_BM) ||
        !make_map(&mbh, Bh, K, n_pad, BN) || !make_map(&mbl, Bl, k_lo, n_pad, BN))
        return cudaErrorInvalidValue;
    constexpr int STAGE_BYTES = 2 * TC_A_BYTES + 2 * BN * TC_BK * 2;
    const size_t smem = (size_t)STAGES * STAGE_BYTES + 256 + 1024;
    auto kern = tc_topk_kernel<BN, STAGES>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, TC_THREADS, smem, st>>>(mah, mal, mbh, mbl, K, k_lo / TC_BK, m_dev,
                                         (unsigned)(n_pad / BN), n, r1, r2, c1, c2, k, part_d,
                                         part_i, err);
    return cudaGetLastError();
}

}  // namespace

int tc_topk_variants() { return 2; }

cudaError_t launch_bounded_wait_selftest(int *err, long long budget_cycles, cudaStream_t st) {
    bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(err, budget_cycles);
    return cudaGetLastError();
}

cudaError_t launch_tc_topk(int variant, const void *Ah, const void *Al, size_t rows_pad,
                           const void *Bh, const void *Bl, size_t n_pad, int K, int k_lo,
                           const int *m_dev, size_t n, const float *r1, const float *r2,
                           const float *c1, const float *c2, int k, float *part_d, int *part_i,
                           int *err, int grid, cudaStream_t st) {
    if (k < 1 || k > kTopKMax) return cudaErrorInvalidValue;
    if (variant == 1)
        return topk_variant<128, 3>(Ah, Al, rows_pad, Bh, Bl, n_pad, K, k_lo, m_dev, n, r1, r2, c1,
                                    c2, k, part_d, part_i, err, grid, st);
    return topk_variant<256, 2>(Ah, Al, rows_pad, Bh, Bl, n_pad, K, k_lo, m_dev, n, r1, r2, c1, c2,
                                k, part_d, part_i, err, grid, st);
}

cudaError_t launch_topk_merge(const int *m_dev, int grid_ctas, const float *part_d,
                              const int *part_i, int k, size_t max_rows, float *out_d,
                              long long *out_i, cudaStream_t st) {
    const int wpb = 8;
    const unsigned blocks = (unsigned)((max_rows + wpb - 1) / wpb);
    topk_merge_kernel<<<blocks ? blocks : 1, 32 * wpb, 0, st>>>(m_dev, grid_ctas, grid_ctas, part_d,
                                                                part_i, k, out_d, out_i);
    return cudaGetLastError();
}

cudaError_t launch_tc_dist(const void *Ah, const void *Al, const void *Bh, const void *Bl, int K,
                           int k_lo, size_t m, size_t m_pad, size_t n, size_t n_pad,
                           const float *r1, const float *r2, const float *c1, const float *c2,
                           float *out, size_t ldo, int *err, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    if (K % TC_BK || k_lo % TC_BK || k_lo <= 0 || k_lo > K || m_pad % TC_BM || n_pad % TC_BN)
        return cudaErrorInvalidValue;
    // TMA: 16-byte aligned bases and row strides
    for (const void *p : {Ah, Al, Bh, Bl})
        if (reinterpret_cast<uintptr_t>(p) & 15) return cudaErrorMisalignedAddress;
    alignas(64) CUtensorMap mah, mal, mbh, mbl;
    if (!make_map(&mah, Ah, K, m_pad, TC_BM) || !make_map(&mal, Al, K, m_pad, TC_BM) ||
        !make_map(&mbh, Bh, K, n_pad, TC_BN) || !make_map(&mbl, Bl, k_lo, n_pad, TC_BN))
        return cudaErrorInvalidValue;
    const size_t smem = (size_t)TC_STAGES * TC_STAGE_BYTES + 256 + 1024;
    cudaError_t e = cudaFuncSetAttribute(tc_dist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const unsigned num_mb = (unsigned)(m_pad / TC_BM);
    const size_t tiles = (size_t)num_mb * (n_pad / TC_BN);
    if (tiles > 0xFFFFFFFFull) return cudaErrorInvalidValue;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)(tiles < (size_t)sms ? tiles : (size_t)sms);
    tc_dist_kernel<<<grid, TC_THREADS, smem, st>>>(mah, mal, mbh, mbl, K, k_lo / TC_BK, num_mb,
                                                   (unsigned)tiles, m, n, r1, r2, c1, c2, out, ldo,
                                                   err);
    return cudaGetLastError();
}

}  // namespace tq
