// tq_tc.cu -- the tensor-core contractions of the M x N distances on sm_100a
// (tcgen05 + TMA), with their epilogues fused: the split-BF16 asymmetric and
// symmetric distances (tc_dist), their per-row top-k over a device-resident
// index (tc_topk, the serving kernel) and the split-TF32 QJL-corrected
// symmetric distances (tc_symq).
//
// C = Ah Bh^T + Ah Bl^T + Al Bh^T over hi/lo operand planes (x = hi + lo,
// see tq_mton.cu and tq_symq.cu), accumulated in FP32 in tensor memory.  A
// product is skipped where its lo operand is zero by construction: B's lo
// from K block kbx on (the +-1 QJL half of asymmetric planes), A's lo in a
// segment marked a_exact (the +-1 signs of the light variant).
//
// Accumulation with promotion.  The tensor core's FP32 accumulation loses
// low bits of what it adds to a large running sum, always toward zero, so a
// reduction whose terms share a sign (a code against itself: squares of
// centroid values) drifted by 1.3e-5 of the result at K = 2048 (measured).
// Here the MMAs of a chunk of CH K blocks accumulate from zero into one of two
// chunk buffers X0 / X1 in tensor memory; the epilogue warps add each chunk
// into a running sum Y (one per K segment, also in tensor memory) with IEEE
// FP32 adds while the MMAs fill the other buffer.  In each K step the small
// products (hi x lo, lo x hi) are issued before hi x hi.  The drift is then
// that of one chunk (CH = 2 K blocks) at any K.
//
// Persistent kernel, one CTA per SM, 10 warps (6 for two K segments), 128 x 128 tiles:
//   warp 0      TMA producer: per K block (128 bytes of K: 64 BF16 or 32
//               TF32 values) loads the Ah, Al, Bh, Bl tiles it needs,
//               128-byte swizzled, into a ring of STAGES stages
//   warp 1      allocates 512 tensor-memory columns (X0, X1, Y0, Y1, 128
//               each); one thread issues the tcgen05.mma of each K block as
//               its stage lands, into the current chunk's buffer, and commits
//               the stage's "empty" barrier and, per chunk, the buffer's
//               "full" barrier
//   warps 2..5  promotion: per chunk, tcgen05.ld the buffer, add it into the
//               running sum Y with tcgen05.ld / st, release the buffer
//   warps 6..9  per tile, the policy's epilogue (distances, top-k) reads Y,
//               double-buffered over tiles; with two K segments (the
//               QJL-corrected distances, Y0 and Y1 per tile) warps 2..5 run
//               it themselves after the tile's promotions
// Every mbarrier wait is bounded: after ~2 s it records an error code in
// *err and the CTA winds down (frees its tensor memory) instead of waiting
// forever.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "tq_async.cuh"
#include "tq_mton.h"

namespace tq {
namespace {

constexpr int TC_BM = 128, TC_BN = 128;
constexpr int TC_BK = 64;    // BF16 values per K block (128 bytes)
constexpr int SQ_TBK = 32;   // TF32 values per K block (128 bytes)
constexpr int TC_A_BYTES = TC_BM * 128;  // 16 KB
constexpr int TC_B_BYTES = TC_BN * 128;  // 16 KB
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;  // 64 KB
constexpr int TC_TMEM_COLS = 512;
// threads: producer, MMA and 4 epilogue warps; plus 4 finalize warps when the
// running sum is double-buffered (one K segment); plus 4 decoder warps when the
// B tiles are decoded from codes in shared memory (DEC)
constexpr int tc_threads(bool split, bool dec = false) { return (split ? 320 : 192) + (dec ? 128 : 0); }
// shared bytes after the stages: barriers and the tensor-memory slot; the DEC
// kernels' decode tables follow (tabc: 256 x 8 B, tabs: 256 x 4 B)
constexpr int TC_BAR_BYTES = 256;
constexpr int TC_DEC_TAB_BYTES = 256 * 8 + 256 * 4;
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
// rows are 128 bytes and whose 8-row groups are 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);  // start address
    d |= (uint64_t)1u << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;        // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                  // layout: SWIZZLE_128B
    return d;
}

// Instruction descriptor: FP32 accumulator, A and B of format `fmt` (1 =
// BF16 for kind::f16, 2 = TF32 for kind::tf32), both K-major, M128 N128.
constexpr uint32_t tc_idesc(uint32_t fmt) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
           ((uint32_t)(TC_BM >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    if constexpr (TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(tc_idesc(2)), "r"(acc)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(tc_idesc(1)), "r"(acc)
            : "memory");
    }
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

// 32 consecutive 32-bit columns of this warp's 32 tensor-memory lanes; the
// _nw form leaves the wait (tcgen05.wait::ld) to the caller.
__device__ __forceinline__ void tmem_ld32_nw(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
// 16 consecutive 32-bit columns of this warp's lanes; the caller waits
// (tcgen05.wait::ld) before reading them.
__device__ __forceinline__ void tmem_ld16_nw(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
        "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
        "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
        "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
        "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
        "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// The tensor maps of up to two K segments: [segment][Ah, Al, Bh, Bl].
struct TcMaps {
    CUtensorMap m[2][4];
};

// K blocks of each segment, the first block whose B lo is zero (kbx = KB: none),
// whether the segment's A lo is zero, and whether its sums are exact in one
// accumulator (whole: products of +-1 by +-1, integer partial sums of
// magnitude <= K < 2^24, which FP32 accumulation holds exactly; the segment
// is then one chunk with no promotion).
struct TcShape {
    int nseg;
    int KB[2], kbx[2], a_exact[2], whole[2];
};

// End of the promoted chunk that starts at K block c0: CH blocks, the
// segment's end, or the end of the centroid half (DEC, asymmetric).
__device__ __forceinline__ int chunk_end(int c0, int chl, int KB, int kbc) {
    int c1 = c0 + chl < KB ? c0 + chl : KB;
    if (c0 < kbc && c1 > kbc) c1 = kbc;
    return c1;
}

// ---------------------------------------------------------------------------
// The pipeline.  Epi supplies the tile schedule (tiles(), tile_at()) and the
// epilogue State (tile() reads the running sums Y0 / Y1 of a finished tile,
// finish() runs once after the last tile).
// SPLIT (one K segment): the running sum is double-buffered over tiles (tile t
// in Y[t & 1]) and 4 more warps (6..9) run the tile epilogue, so that it
// overlaps the next tile's MMAs and promotions; the promotion warps then wait
// for Y[t & 1] to be read ("yempty") and signal it complete ("yfull").
// Otherwise (two segments, Y0 and Y1 per tile) warps 2..5 do both.
// ---------------------------------------------------------------------------
template <bool TF32, int STAGES, int CH, bool SPLIT, class Epi, bool DEC = false>
__global__ void __launch_bounds__(tc_threads(SPLIT, DEC), 1) tcp_kernel(const __grid_constant__ TcMaps maps,
                                                                        const TcShape sh,
                                                                        const typename Epi::Params ep,
                                                                        int *err, const DecSrc dec) {
    static_assert(!DEC || (!TF32 && SPLIT), "decoded B tiles: BF16, one K segment");
    constexpr int KBLK = TF32 ? SQ_TBK : TC_BK;  // values per K block
    extern __shared__ unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled tiles
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * TC_STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], xfull[2], xempty[2], drain, yfull[2],
    // yempty[2]; then the TMEM slot
    // DEC: cfull[2], cempty[2] (code tile buffers) follow; then the TMEM slot
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 9 + (DEC ? 4 : 0));
    const uint32_t cfull0 = smem_u32(bars + 2 * STAGES + 9), cempty0 = cfull0 + 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
    const uint32_t xfull0 = smem_u32(bars + 2 * STAGES), xempty0 = smem_u32(bars + 2 * STAGES + 2);
    const uint32_t drain = smem_u32(bars + 2 * STAGES + 4);
    const uint32_t yfull0 = smem_u32(bars + 2 * STAGES + 5), yempty0 = smem_u32(bars + 2 * STAGES + 7);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, DEC ? 1 + 128 : 1);  // DEC: the producer and 128 decoders
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(xfull0 + 8 * b, 1);
            mbar_init(xempty0 + 8 * b, 128);
            mbar_init(yfull0 + 8 * b, 128);
            mbar_init(yempty0 + 8 * b, 128);
        }
        mbar_init(drain, 1);
        if constexpr (DEC) {
            for (int b = 0; b < 2; ++b) {
                mbar_init(cfull0 + 8 * b, 1);
                mbar_init(cempty0 + 8 * b, 128);
            }
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // DEC decode tables: nibble codes: tabc[byte] = {hi pair, lo pair} of its
    // two units' centroids, tabs[byte] = their +-1 pair; byte codes: tabc as
    // 256 words hi | lo << 16 of c[u >> 1].
    uint2 *tabc = reinterpret_cast<uint2 *>(smem + STAGES * TC_STAGE_BYTES + TC_BAR_BYTES);
    uint32_t *tabs = reinterpret_cast<uint32_t *>(tabc + 256);
    if constexpr (DEC) {
        auto cpair = [&](unsigned u, uint32_t &h, uint32_t &l) {
            const unsigned v = u >> 1;
            const float c = v < (unsigned)dec.levels ? dec.centroids[v] : 0.0f;
            const __nv_bfloat16 hb = __float2bfloat16_rn(c);
            const __nv_bfloat16 lb = __float2bfloat16_rn(c - __bfloat162float(hb));
            h = __bfloat16_as_ushort(hb);
            l = __bfloat16_as_ushort(lb);
        };
        for (int i = threadIdx.x; i < 256; i += blockDim.x) {
            uint32_t h0, l0, h1, l1;
            if (dec.nibble) {
                cpair(i & 15, h0, l0);
                cpair(i >> 4, h1, l1);
                tabc[i] = make_uint2(h0 | (h1 << 16), l0 | (l1 << 16));
                tabs[i] = ((i & 1) ? 0x3F80u : 0xBF80u) | (((i & 16) ? 0x3F80u : 0xBF80u) << 16);
            } else {
                cpair(i, h0, l0);
                reinterpret_cast<uint32_t *>(tabc)[i] = h0 | (l0 << 16);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int ntiles = Epi::tiles(ep);

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int t = 0; t < ntiles && ok; ++t) {
                int mb, nb;
                Epi::tile_at(ep, t, mb, nb);
                for (int sg = 0; sg < sh.nseg && ok; ++sg) {
                    const CUtensorMap *mp = maps.m[sg];
                    const bool alo = !sh.a_exact[sg];
                    for (int kb = 0; kb < sh.KB[sg]; ++kb, ++it) {
                        const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err, kErrEmpty)) { ok = false; break; }
                        const bool blo = kb < sh.kbx[sg];
                        const uint32_t base = smem_u32(smem + s * TC_STAGE_BYTES);
                        const uint32_t fb = full0 + 8 * s;
                        const int kx = kb * KBLK;
                        if constexpr (DEC) {  // B comes from the decoder warps
                            mbar_expect_tx(fb, (alo ? 2 : 1) * TC_A_BYTES);
                            tma_load_2d(base, &mp[0], kx, mb * TC_BM, fb);
                            if (alo) tma_load_2d(base + TC_A_BYTES, &mp[1], kx, mb * TC_BM, fb);
                        } else {
                            mbar_expect_tx(fb, (alo ? 2 : 1) * TC_A_BYTES + (blo ? 2 : 1) * TC_B_BYTES);
                            tma_load_2d(base, &mp[0], kx, mb * TC_BM, fb);
                            if (alo) tma_load_2d(base + TC_A_BYTES, &mp[1], kx, mb * TC_BM, fb);
                            tma_load_2d(base + 2 * TC_A_BYTES, &mp[2], kx, nb * TC_BN, fb);
                            if (blo) tma_load_2d(base + 2 * TC_A_BYTES + TC_B_BYTES, &mp[3], kx, nb * TC_BN, fb);
                        }
                    }
                }
            }
            // every stage issued must have landed before the CTA exits
            for (uint32_t k = 0; k < (uint32_t)STAGES && k < it; ++k) {
                const uint32_t j = it - 1 - k;
                mbar_drain(full0 + 8 * (j % STAGES), (j / STAGES) & 1u);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t it = 0, gc = 0;
            bool ok = true;
            for (int t = 0; t < ntiles && ok; ++t) {
                for (int sg = 0; sg < sh.nseg && ok; ++sg) {
                    const bool alo = !sh.a_exact[sg];
                    const int chl = sh.whole[sg] ? sh.KB[sg] : CH;
                    const int kbc = DEC ? dec.kbc : sh.KB[sg];
                    for (int c0 = 0, c1 = 0; c0 < sh.KB[sg] && ok; c0 = c1, ++gc) {
                        c1 = chunk_end(c0, chl, sh.KB[sg], kbc);
                        const uint32_t b = gc & 1u, xph = (gc >> 1) & 1u;
                        if (!mbar_wait(xempty0 + 8 * b, xph ^ 1u, err, kErrTmemEmpty)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t d_tmem = tmem_base + b * TC_BN;
                        uint32_t acc = 0u;
                        for (int kb = c0; kb < c1; ++kb, ++it) {
                            const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                            if (!mbar_wait(full0 + 8 * s, ph, err, kErrFull)) { ok = false; break; }
                            tc_fence_after();
                            const bool blo = kb < sh.kbx[sg];
                            const uint32_t base = smem_u32(smem + s * TC_STAGE_BYTES);
                            const uint32_t ah = base, al = base + TC_A_BYTES;
                            const uint32_t bh = base + 2 * TC_A_BYTES, bl = bh + TC_B_BYTES;
#pragma unroll
                            for (int kk = 0; kk < 4; ++kk) {
                                const uint32_t koff = kk * 32;  // one MMA's K: 32 bytes
                                // the small products first, while the sum is smaller
                                if (blo) {
                                    umma<TF32>(d_tmem, sw128_desc(ah + koff), sw128_desc(bl + koff), acc);
                                    acc = 1u;
                                }
                                if (alo) {
                                    umma<TF32>(d_tmem, sw128_desc(al + koff), sw128_desc(bh + koff), acc);
                                    acc = 1u;
                                }
                                umma<TF32>(d_tmem, sw128_desc(ah + koff), sw128_desc(bh + koff), acc);
                                acc = 1u;
                            }
                            umma_commit(empty0 + 8 * s);  // stage free once these MMAs are done
                        }
                        if (ok) umma_commit(xfull0 + 8 * b);  // chunk sum ready
                    }
                }
            }
            // every MMA issued must be complete before the tensor memory is freed
            umma_commit(drain);
            mbar_drain(drain, 0);
        }
    } else if (!SPLIT || warp < 6) {
        // ---------------- promotion (warps 2..5, 128 threads) ----------------
        // (without SPLIT these warps also run the tile epilogue)
        const int q = warp & 3;  // the tensor-memory lane quadrant this warp may access
        const uint32_t lanes = tmem_base + ((uint32_t)(32 * q) << 16);
        typename Epi::State st(ep, 32 * q + lane);
        uint32_t gc = 0;
        bool ok = true;
        for (int t = 0; t < ntiles && ok; ++t) {
            const uint32_t yb = (uint32_t)t & 1u, yph = ((uint32_t)t >> 1) & 1u;
            if constexpr (SPLIT) {
                if (!mbar_wait(yempty0 + 8 * yb, yph ^ 1u, err, kErrTmemEmpty)) { ok = false; break; }
                tc_fence_after();
            }
            int mb_t = 0, nb_t = 0;
            if constexpr (DEC) Epi::tile_at(ep, t, mb_t, nb_t);
            for (int sg = 0; sg < sh.nseg && ok; ++sg) {
                const uint32_t Y = lanes + (2 + (SPLIT ? yb : (uint32_t)sg)) * TC_BN;
                const int chl = sh.whole[sg] ? sh.KB[sg] : CH;
                const int kbc = DEC ? dec.kbc : sh.KB[sg];
                for (int c0 = 0, c1 = 0; c0 < sh.KB[sg]; c0 = c1, ++gc) {
                    c1 = chunk_end(c0, chl, sh.KB[sg], kbc);
                    const uint32_t b = gc & 1u, xph = (gc >> 1) & 1u;
                    if (!mbar_wait(xfull0 + 8 * b, xph, err, kErrTmemFull)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t X = lanes + b * TC_BN;
                    // DEC: this chunk's per-column factor (centroid or sign half)
                    const float *fsrc = nullptr;
                    if constexpr (DEC) fsrc = dec.fc ? (c0 < dec.kbc ? dec.fc : dec.fs) : nullptr;
#pragma unroll 1
                    for (int p = 0; p < TC_BN / 32; ++p) {
                        uint32_t x[32], y[32];
                        __syncwarp();
                        tmem_ld32_nw(X + 32 * p, x);
                        if (c0 != 0) tmem_ld32_nw(Y + 32 * p, y);
                        tmem_wait_ld();
                        if (DEC && fsrc) {
                            const float *f = fsrc + (size_t)nb_t * TC_BN + 32 * p;
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const float xv = __uint_as_float(x[j]), fj = __ldg(f + j);
                                x[j] = __float_as_uint(c0 != 0 ? __fmaf_rn(xv, fj, __uint_as_float(y[j]))
                                                               : __fmul_rn(xv, fj));
                            }
                        } else if (c0 != 0) {
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                x[j] = __float_as_uint(__fadd_rn(__uint_as_float(y[j]), __uint_as_float(x[j])));
                        }
                        tmem_st32(Y + 32 * p, x);
                    }
                    tmem_wait_st();
                    __syncwarp();
                    tc_fence_before();
                    mbar_arrive(xempty0 + 8 * b);
                }
            }
            if (!ok) break;
            if constexpr (SPLIT) {
                mbar_arrive(yfull0 + 8 * yb);  // Y[yb] complete (its stores were waited for)
            } else {
                int mb, nb;
                Epi::tile_at(ep, t, mb, nb);
                st.tile(ep, mb, nb, lanes + 2 * TC_BN, lanes + 3 * TC_BN);
            }
        }
        if constexpr (!SPLIT) {
            if (ok) st.finish(ep);
        }
    } else if (!DEC || warp < 10) {
        // ---------------- tile epilogue (warps 6..9, SPLIT only) ----------------
        const int q = warp & 3;
        const uint32_t lanes = tmem_base + ((uint32_t)(32 * q) << 16);
        typename Epi::State st(ep, 32 * q + lane);
        bool ok = true;
        for (int t = 0; t < ntiles; ++t) {
            const uint32_t yb = (uint32_t)t & 1u, yph = ((uint32_t)t >> 1) & 1u;
            if (!mbar_wait(yfull0 + 8 * yb, yph, err, kErrTmemFull)) { ok = false; break; }
            tc_fence_after();
            int mb, nb;
            Epi::tile_at(ep, t, mb, nb);
            st.tile(ep, mb, nb, lanes + (2 + yb) * TC_BN, 0u);
            __syncwarp();
            tc_fence_before();
            mbar_arrive(yempty0 + 8 * yb);
        }
        if (ok) st.finish(ep);
    } else if constexpr (DEC) {
        // ---------------- decoders (warps 10..13, DEC only) ----------------
        // Each tile's 128 codes arrive in shared memory as one bulk copy
        // (dec.cbufs buffers: the next tile's copy is in flight while this one
        // is decoded).  Thread r writes row r of each B tile (code nb * 128 +
        // r): eight 16-byte chunks of 8 values, chunk w at (w ^ (r & 7)) * 16
        // of the row's 128 bytes (the TMA's 128-byte swizzle).  Thread 0 issues
        // the copies; a buffer is reused once all 128 threads have arrived on
        // its cempty barrier.
        const int r = threadIdx.x - 320, sw = r & 7;
        const int wpb = dec.nibble ? 8 : 16;  // code words per K block
        const int KB = sh.KB[0];
        const int nbuf = dec.cbufs;
        const uint32_t tile_bytes = (uint32_t)dec.ctile_bytes;
        unsigned char *cbuf0 = reinterpret_cast<unsigned char *>(tabs + 256);
        // copy of tile tt's codes into buffer bb (rows past n: whatever lies beyond
        // the corpus in its allocation, which is padded to 256 bytes; unused)
        auto issue = [&](int tt, int bb) {
            int mb, nb;
            Epi::tile_at(ep, tt, mb, nb);
            const size_t j0 = (size_t)nb * TC_BN;
            const size_t rows = dec.n - j0 < (size_t)TC_BN ? dec.n - j0 : (size_t)TC_BN;
            const uint32_t bytes = ((uint32_t)(rows * (size_t)dec.cs) + 15u) & ~15u;
            const uint32_t bar = cfull0 + 8 * bb;
            mbar_expect_tx(bar, bytes);
            bulk_load(smem_u32(cbuf0 + (size_t)bb * tile_bytes), dec.codes + j0 * (size_t)dec.cs, bytes, bar);
        };
        uint32_t it = 0;
        bool ok = true;
        int issued = 0, waited = 0;  // tiles whose copy thread 0 issued / saw land
        if (r == 0 && ntiles > 0) {
            issue(0, 0);
            issued = 1;
        }
        for (int t = 0; t < ntiles && ok; ++t) {
            const int bb = nbuf == 2 ? (t & 1) : 0;
            const uint32_t use = nbuf == 2 ? (uint32_t)(t >> 1) : (uint32_t)t;  // uses of bb before
            if (r == 0 && nbuf == 2 && t + 1 < ntiles) {
                // the other buffer is free once tile t - 1 was decoded
                if (t >= 1 && !mbar_wait(cempty0 + 8 * ((t + 1) & 1), (uint32_t)((t - 1) >> 1) & 1u, err,
                                         kErrEmpty)) {
                    ok = false;
                    break;
                }
                issue(t + 1, (t + 1) & 1);
                issued = t + 2;
            }
            if (!mbar_wait(cfull0 + 8 * bb, use & 1u, err, kErrFull)) { ok = false; break; }
            waited = t + 1;
            int mb, nb;
            Epi::tile_at(ep, t, mb, nb);
            const bool live = (unsigned)nb * TC_BN + (unsigned)r < dec.n;
            const uint32_t *crow = reinterpret_cast<const uint32_t *>(cbuf0 + (size_t)bb * tile_bytes +
                                                                      (size_t)r * (size_t)dec.cs);
            for (int kb = 0; kb < KB; ++kb, ++it) {
                const bool cent = kb < dec.kbc;
                const int kq = cent ? kb : kb - dec.kbc;  // K block within its half
                uint32_t w[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) w[i] = (live && i < wpb) ? crow[kq * wpb + i] : 0u;
                if (kb == KB - 1) mbar_arrive(cempty0 + 8 * bb);  // this thread is done with the tile
                const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err, kErrEmpty)) { ok = false; break; }
                unsigned char *bh = smem + s * TC_STAGE_BYTES + 2 * TC_A_BYTES + r * 128;
                unsigned char *bl = bh + TC_B_BYTES;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    uint4 hi = make_uint4(0u, 0u, 0u, 0u), lo = hi;
                    if (live) {
                        if (dec.nibble) {
                            const uint32_t x = w[c];
                            uint32_t hv[4], lv[4];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const uint32_t byte = (x >> (8 * q)) & 0xFFu;
                                if (cent) {
                                    const uint2 e = tabc[byte];
                                    hv[q] = e.x;
                                    lv[q] = e.y;
                                } else {
                                    hv[q] = tabs[byte];
                                    lv[q] = 0u;
                                }
                            }
                            hi = make_uint4(hv[0], hv[1], hv[2], hv[3]);
                            lo = make_uint4(lv[0], lv[1], lv[2], lv[3]);
                        } else {
                            const uint32_t *t1 = reinterpret_cast<const uint32_t *>(tabc);
                            uint32_t hv[4], lv[4];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const uint32_t x = w[2 * c + (q >> 1)];
                                const uint32_t u0 = (x >> (16 * (q & 1))) & 0xFFu;
                                const uint32_t u1 = (x >> (16 * (q & 1) + 8)) & 0xFFu;
                                if (cent) {
                                    const uint32_t e0 = t1[u0], e1 = t1[u1];
                                    hv[q] = __byte_perm(e0, e1, 0x5410u);
                                    lv[q] = __byte_perm(e0, e1, 0x7632u);
                                } else {
                                    hv[q] = ((u0 & 1u) ? 0x3F80u : 0xBF80u) |
                                            (((u1 & 1u) ? 0x3F80u : 0xBF80u) << 16);
                                    lv[q] = 0u;
                                }
                            }
                            hi = make_uint4(hv[0], hv[1], hv[2], hv[3]);
                            lo = make_uint4(lv[0], lv[1], lv[2], lv[3]);
                        }
                    }
                    const int off = (c ^ sw) << 4;
                    *reinterpret_cast<uint4 *>(bh + off) = hi;
                    if (kb < sh.kbx[0]) *reinterpret_cast<uint4 *>(bl + off) = lo;
                }
                fence_proxy_async_smem();  // the tile's generic stores before the MMA's async reads
                mbar_arrive(full0 + 8 * s);
            }
            if (ok && r == 0 && nbuf == 1 && t + 1 < ntiles) {
                // one buffer: the next tile's copy once every thread read this one
                if (!mbar_wait(cempty0, (uint32_t)t & 1u, err, kErrEmpty)) { ok = false; break; }
                issue(t + 1, 0);
                issued = t + 2;
            }
        }
        if (r == 0) {
            // the copies issued but not seen to land must do so before the CTA exits
            for (int tt = waited; tt < issued; ++tt) {
                const int bb = nbuf == 2 ? (tt & 1) : 0;
                const uint32_t use = nbuf == 2 ? (uint32_t)(tt >> 1) : (uint32_t)tt;
                mbar_drain(cfull0 + 8 * bb, use & 1u);
            }
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

// Reads 32 columns of a running sum as floats.
__device__ __forceinline__ void ld_sum32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    __syncwarp();
    tmem_ld32(taddr, r);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// ---- epilogue policies --------------------------------------------------------
// Tiles of an m_pad x n_pad output visited with the row-block index fastest,
// so that CTAs running at the same time share the B tile in L2.
struct GridTiles {
    unsigned num_mb, num_tiles;
    __device__ static int count(unsigned num_tiles) {
        return blockIdx.x < num_tiles ? (int)((num_tiles - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
    }
    __device__ void at(int t, int &mb, int &nb) const {
        const unsigned tile = blockIdx.x + (unsigned)t * gridDim.x;
        mb = (int)(tile % num_mb);
        nb = (int)(tile / num_mb);
    }
};

// d = max(0, r2_i + c2_j - 2 (C_ij r1_i) c1_j), stored to out[i * ldo + j].
struct DistEpi {
    struct Params {
        GridTiles g;
        size_t m, n;
        const float *r1, *r2, *c1, *c2;
        float *out;
        size_t ldo;
    };
    __device__ static int tiles(const Params &p) { return GridTiles::count(p.g.num_tiles); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) { p.g.at(t, mb, nb); }
    struct State {
        int rit;
        bool vec;
        __device__ State(const Params &p, int row_in_tile)
            : rit(row_in_tile),
              vec(((p.ldo & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.out) & 15) == 0)) {}
        __device__ void tile(const Params &p, int mb, int nb, uint32_t y0, uint32_t) {
            const size_t row = (size_t)mb * TC_BM + rit;
            const bool row_ok = row < p.m;
            const float rr1 = row_ok ? __ldg(p.r1 + row) : 0.0f;
            const float rr2 = row_ok ? __ldg(p.r2 + row) : 0.0f;
            float *orow = p.out + row * p.ldo;
#pragma unroll 1
            for (int ch = 0; ch < TC_BN / 32; ++ch) {
                float c[32];
                ld_sum32(y0 + 32 * ch, c);
                const size_t col0 = (size_t)nb * TC_BN + ch * 32;
                if (!row_ok || col0 >= p.n) continue;
                float dv[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const size_t col = col0 + j < p.n ? col0 + j : p.n - 1;
                    const float ipt = __fmul_rn(__fmul_rn(c[j], rr1), __ldg(p.c1 + col));
                    const float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + col)), __fmul_rn(2.0f, ipt));
                    dv[j] = d > 0.0f ? d : 0.0f;
                }
                if (vec && col0 + 32 <= p.n) {
                    float4 *o4 = reinterpret_cast<float4 *>(orow + col0);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        o4[j] = make_float4(dv[4 * j], dv[4 * j + 1], dv[4 * j + 2], dv[4 * j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (col0 + j < p.n) orow[col0 + j] = dv[j];
                }
            }
        }
        __device__ void finish(const Params &) {}
    };
};

// ---------------------------------------------------------------------------
// tcw_kernel: the M x N distances and the serving top-k with 128 x 256 tiles
// (epilogue policies WDist, WTopk).  A 128 x 128 tile
// with three operand reads per K step needs more shared-memory bandwidth than
// the SM has once the TMA writes are counted (128 B/clk of MMA operands + 85
// B/clk of copies), which held tcp_kernel near half of the tensor cycles; a
// 256-wide tile needs 96 + 62.5 B/clk.  The two 256-column chunk buffers then
// fill the tensor memory, so the running sum lives in registers: 8 epilogue
// warps, two per lane quadrant, each thread one row and 128 of the columns.
// The promotion loads a chunk in 16-column pieces, the next piece in flight
// while the current one is added, so that the MMAs seldom wait for a chunk
// buffer; the distances are written from the registers.  Otherwise as
// tcp_kernel (promoted chunks of CH K blocks, bounded waits).
// ---------------------------------------------------------------------------
constexpr int TW_BN = 256;
constexpr int TW_B_BYTES = TW_BN * 128;                           // 32 KB
constexpr int TW_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TW_B_BYTES;  // 96 KB
constexpr int TW_EPI_WARPS = 8, TW_COLS = TW_BN * 4 / TW_EPI_WARPS;  // 128 columns per thread
constexpr int TW_THREADS = 32 * (2 + TW_EPI_WARPS);
constexpr uint32_t kIdescW = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TW_BN >> 3) << 17) |
                             ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ void umma_w(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdescW), "r"(acc)
        : "memory");
}

template <int STAGES, int CH, class W>
__global__ void __launch_bounds__(TW_THREADS, 1) tcw_kernel(const __grid_constant__ TcMaps maps,
                                                            const TcShape sh,
                                                            const typename W::Params ep, int *err) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + STAGES * TW_STAGE_BYTES);
    // bars: full[STAGES], empty[STAGES], xfull[2], xempty[2], drain; then the TMEM slot
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 5);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);
    const uint32_t xfull0 = smem_u32(bars + 2 * STAGES), xempty0 = smem_u32(bars + 2 * STAGES + 2);
    const uint32_t drain = smem_u32(bars + 2 * STAGES + 4);
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(xfull0 + 8 * b, 1);
            mbar_init(xempty0 + 8 * b, 32 * TW_EPI_WARPS);
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
    const int ntiles = W::tiles(ep);
    const int KB = sh.KB[0], kbx = sh.kbx[0];
    const CUtensorMap *mp = maps.m[0];

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int t = 0; t < ntiles && ok; ++t) {
                int mb, nb;
                W::tile_at(ep, t, mb, nb);
                for (int kb = 0; kb < KB; ++kb, ++it) {
                    const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                    if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err, kErrEmpty)) { ok = false; break; }
                    const bool blo = kb < kbx;
                    const uint32_t base = smem_u32(smem + s * TW_STAGE_BYTES);
                    const uint32_t fb = full0 + 8 * s;
                    mbar_expect_tx(fb, 2 * TC_A_BYTES + (blo ? 2 : 1) * TW_B_BYTES);
                    const int kx = kb * TC_BK;
                    tma_load_2d(base, &mp[0], kx, mb * TC_BM, fb);
                    tma_load_2d(base + TC_A_BYTES, &mp[1], kx, mb * TC_BM, fb);
                    tma_load_2d(base + 2 * TC_A_BYTES, &mp[2], kx, nb * TW_BN, fb);
                    if (blo) tma_load_2d(base + 2 * TC_A_BYTES + TW_B_BYTES, &mp[3], kx, nb * TW_BN, fb);
                }
            }
            for (uint32_t k = 0; k < (uint32_t)STAGES && k < it; ++k) {
                const uint32_t j = it - 1 - k;
                mbar_drain(full0 + 8 * (j % STAGES), (j / STAGES) & 1u);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t it = 0, gc = 0;
            bool ok = true;
            for (int t = 0; t < ntiles && ok; ++t) {
                for (int c0 = 0; c0 < KB && ok; c0 += CH, ++gc) {
                    const uint32_t b = gc & 1u, xph = (gc >> 1) & 1u;
                    if (!mbar_wait(xempty0 + 8 * b, xph ^ 1u, err, kErrTmemEmpty)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + b * TW_BN;
                    const int c1 = c0 + CH < KB ? c0 + CH : KB;
                    uint32_t acc = 0u;
                    for (int kb = c0; kb < c1; ++kb, ++it) {
                        const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
                        if (!mbar_wait(full0 + 8 * s, ph, err, kErrFull)) { ok = false; break; }
                        tc_fence_after();
                        const bool blo = kb < kbx;
                        const uint32_t base = smem_u32(smem + s * TW_STAGE_BYTES);
                        const uint32_t ah = base, al = base + TC_A_BYTES;
                        const uint32_t bh = base + 2 * TC_A_BYTES, bl = bh + TW_B_BYTES;
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            const uint32_t koff = kk * 32;
                            if (blo) {
                                umma_w(d_tmem, sw128_desc(ah + koff), sw128_desc(bl + koff), acc);
                                acc = 1u;
                            }
                            umma_w(d_tmem, sw128_desc(al + koff), sw128_desc(bh + koff), acc);
                            umma_w(d_tmem, sw128_desc(ah + koff), sw128_desc(bh + koff), 1u);
                            acc = 1u;
                        }
                        umma_commit(empty0 + 8 * s);
                    }
                    if (ok) umma_commit(xfull0 + 8 * b);
                }
            }
            umma_commit(drain);
            mbar_drain(drain, 0);
        }
    } else {
        // ---------------- epilogue (warps 2..9, 256 threads) ----------------
        const int q = warp & 3, h = (warp - 2) >> 2;  // lane quadrant, column half
        const uint32_t lanes = tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(TW_COLS * h);
        typename W::State st(ep, 32 * q + lane, h);
        if constexpr (W::kDirect) {
            // one chunk per tile (CH >= KB): the tile's sums are read in place
            bool ok = true;
            for (int t = 0; t < ntiles && ok; ++t) {
                int mb, nb;
                W::tile_at(ep, t, mb, nb);
                const uint32_t b = (uint32_t)t & 1u, xph = ((uint32_t)t >> 1) & 1u;
                if (!mbar_wait(xfull0 + 8 * b, xph, err, kErrTmemFull)) { ok = false; break; }
                tc_fence_after();
                st.tile_tmem(ep, mb, nb, lanes + b * TW_BN);
                __syncwarp();
                tc_fence_before();
                mbar_arrive(xempty0 + 8 * b);
            }
            if (ok) st.finish(ep);
        } else {
        float y[TW_COLS];
        uint32_t gc = 0;
        bool ok = true;
        for (int t = 0; t < ntiles && ok; ++t) {
            int mb, nb;
            W::tile_at(ep, t, mb, nb);
            for (int c0 = 0; c0 < KB; c0 += CH, ++gc) {
                const uint32_t b = gc & 1u, xph = (gc >> 1) & 1u;
                if (!mbar_wait(xfull0 + 8 * b, xph, err, kErrTmemFull)) { ok = false; break; }
                tc_fence_after();
                const uint32_t X = lanes + b * TW_BN;
                uint32_t xa[16], xb[16];
                __syncwarp();
                tmem_ld16_nw(X, xa);
                tmem_wait_ld();
#pragma unroll
                for (int p = 0; p < TW_COLS / 16; ++p) {
                    uint32_t(&cur)[16] = (p & 1) ? xb : xa;
                    uint32_t(&nxt)[16] = (p & 1) ? xa : xb;
                    if (p + 1 < TW_COLS / 16) tmem_ld16_nw(X + 16 * (p + 1), nxt);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float a = __uint_as_float(cur[j]);
                        y[16 * p + j] = c0 == 0 ? a : __fadd_rn(y[16 * p + j], a);
                    }
                    tmem_wait_ld();
                }
                __syncwarp();
                tc_fence_before();
                mbar_arrive(xempty0 + 8 * b);
            }
            if (!ok) break;
            st.tile(ep, mb, nb, y);
        }
        if (ok) st.finish(ep);
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

__device__ __forceinline__ bool better(float d, int i, float bd, int bi) {
    return d < bd || (d == bd && i < bi);
}

struct TopkEntry {
    float d;
    int i;
};

// Inserts (d, ci) into the ascending list (bd, bi) of k >= 1 entries, ties
// broken by the smaller index, and returns its new k-th entry.  Out of line
// and rolled: few columns pass a row's threshold, and a sorted insert inlined
// into every column of the unrolled epilogue loops made their code many times
// larger than the instruction cache.
__device__ __noinline__ TopkEntry topk_insert(float *bd, int *bi, int k, float d, int ci) {
    float cd = d;
    int cx = ci;
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
    return TopkEntry{bd[k - 1], bi[k - 1]};
}

// Inserts (d, i), better than the last entry, into the ascending register
// list (bd, bi) of kCandMax entries (ties broken by the smaller index).  With
// b_u = (d, i) better than entry u, slot u takes entry u - 1 when b_{u-1},
// else (d, i) when b_u, else keeps its entry; each slot reads only old
// entries (slots are rewritten from the last down), so the slots do not form
// a dependency chain.
__device__ __forceinline__ void reg_insert(float (&bd)[kCandMax], int (&bi)[kCandMax], float d, int i) {
    bool bu = true;  // b_{kCandMax-1}: the caller's test
#pragma unroll
    for (int u = kCandMax - 1; u > 0; --u) {
        const bool bl = better(d, i, bd[u - 1], bi[u - 1]);
        const float nd = bl ? bd[u - 1] : (bu ? d : bd[u]);
        const int ni = bl ? bi[u - 1] : (bu ? i : bi[u]);
        bd[u] = nd;
        bi[u] = ni;
        bu = bl;
    }
    if (bu) {
        bd[0] = d;
        bi[0] = i;
    }
}

// Per-row top-k over a device-resident index.  The number of query rows m is
// read from device memory (so that one captured launch serves batches of any
// size up to the buffers' capacity).  CTA c takes row block c / S and the
// contiguous slice c % S of the column tiles, S = grid / row blocks; each
// epilogue thread keeps its row's best k (distance, index) pairs, ties broken
// by the smaller index, and writes them to the partial buffers
// part_d / part_i [(block * S + slice) * 128 + row][kCandMax].
// A candidate as one unsigned key, ordered as (distance, index): distances are
// non-negative (or +inf), so their bit patterns order like the values.
__device__ __forceinline__ unsigned long long topk_key(float d, int i) {
    return ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)i;
}
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

struct TopkEpi {
    struct Params {
        const int *m_dev;
        unsigned nb_tiles;
        size_t n;
        const float *r1, *r2, *c1, *c2;
        int k;
        float *part_d;
        int *part_i;
        // per query row, the smallest last-entry key any epilogue thread of the
        // launch has published (all ones before the launch; nullptr: not kept).
        // A thread's full list proves kCandMax candidates at or below its last
        // entry, so no column above the published minimum can be among the
        // row's best kCandMax: every thread tests its columns against
        // min(own last entry, published), read once per tile (a stale value is
        // only larger), and publishes its own last entry after each tile.
        unsigned long long *gthr;
    };
    // this CTA's row block, column-tile range; false when it has no slice
    __device__ static bool slice(const Params &p, int &mb, unsigned &nb0, unsigned &nb1) {
        const int m = *p.m_dev;
        const int num_mb = (m + TC_BM - 1) / TC_BM;
        if (num_mb <= 0 || num_mb > (int)gridDim.x) return false;
        const int S = (int)gridDim.x / num_mb;
        if ((int)blockIdx.x >= num_mb * S) return false;
        mb = (int)blockIdx.x / S;
        const int sl = (int)blockIdx.x % S;
        nb0 = (unsigned)(((size_t)p.nb_tiles * sl) / S);
        nb1 = (unsigned)(((size_t)p.nb_tiles * (sl + 1)) / S);
        return true;
    }
    __device__ static int tiles(const Params &p) {
        int mb;
        unsigned nb0, nb1;
        return slice(p, mb, nb0, nb1) ? (int)(nb1 - nb0) : 0;
    }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) {
        unsigned nb0, nb1;
        slice(p, mb, nb0, nb1);
        nb = (int)nb0 + t;
    }
    struct State {
        int rit, m;
        bool valid;
        float rr1 = 0.0f, rr2 = 0.0f;
        // the row's best kCandMax entries (ascending): the first p.k of them
        // are its best p.k
        float bd[kCandMax];
        int bi[kCandMax];
        __device__ State(const Params &p, int row_in_tile) : rit(row_in_tile) {
            int mb;
            unsigned nb0, nb1;
            m = *p.m_dev;
            valid = slice(p, mb, nb0, nb1);
            const int row = valid ? mb * TC_BM + rit : 0;
            if (valid && row < m) {
                rr1 = __ldg(p.r1 + row);
                rr2 = __ldg(p.r2 + row);
            }
#pragma unroll
            for (int t = 0; t < kCandMax; ++t) {
                bd[t] = INFINITY;
                bi[t] = 0x7fffffff;
            }
        }
        // Each 16-column chunk: the distances in registers and a mask of the
        // columns that beat the list's last entry; only when some column does,
        // the chunk's distances go to a local array and the marked columns are
        // inserted one by one.  Late in a slice few chunks have any.
        __device__ void tile(const Params &p, int mb, int nb, uint32_t y0, uint32_t) {
            const int row = mb * TC_BM + rit;
            const bool row_ok = row < m;
            const size_t colbase = (size_t)nb * TC_BN;
            const unsigned long long g = (row_ok && p.gthr) ? ld_volatile_u64(p.gthr + row) : ~0ull;
#pragma unroll 1
            for (int ch = 0; ch < TC_BN / 16; ++ch) {
                uint32_t r[16];
                __syncwarp();
                tmem_ld16_nw(y0 + 16 * ch, r);  // warp-collective: every lane loads
                tmem_wait_ld();
                if (!row_ok) continue;
                const size_t col0 = colbase + ch * 16;
                const unsigned long long own = topk_key(bd[kCandMax - 1], bi[kCandMax - 1]);
                const unsigned long long T = own < g ? own : g;
                float c[16];
                uint32_t pass = 0u;
#pragma unroll
                for (int j = 0; j < 16; ++j) {  // c[j] <- the column's distance
                    const size_t col = col0 + j;
                    const size_t cc = col < p.n ? col : p.n - 1;
                    const float ipt = __fmul_rn(__fmul_rn(__uint_as_float(r[j]), rr1), __ldg(p.c1 + cc));
                    float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + cc)), __fmul_rn(2.0f, ipt));
                    d = d > 0.0f ? d : 0.0f;
                    c[j] = d;
                    if (col < p.n && topk_key(d, (int)col) < T) pass |= 1u << j;
                }
                if (pass) {
                    float sd[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) sd[j] = c[j];
                    do {
                        const int j = __ffs(pass) - 1;
                        pass &= pass - 1u;
                        const float d = sd[j];
                        const int ci = (int)(col0 + (size_t)j);
                        const unsigned long long kj = topk_key(d, ci);
                        if (kj < topk_key(bd[kCandMax - 1], bi[kCandMax - 1]) && kj < g)
                            reg_insert(bd, bi, d, ci);
                    } while (pass);
                }
            }
            if (row_ok && p.gthr) {
                const unsigned long long own = topk_key(bd[kCandMax - 1], bi[kCandMax - 1]);
                if (own < g) atomicMin(p.gthr + row, own);
            }
        }
        __device__ void finish(const Params &p) {
            if (!valid) return;
            int mb;
            unsigned nb0, nb1;
            slice(p, mb, nb0, nb1);
            if (mb * TC_BM + rit >= m) return;
            const size_t o = ((size_t)blockIdx.x * TC_BM + rit) * kCandMax;
#pragma unroll
            for (int u = 0; u < kCandMax; ++u)
                if (u < p.k) {
                    p.part_d[o + u] = bd[u];
                    p.part_i[o + u] = bi[u];
                }
        }
    };
};

// The threshold collection of the exact stage's open rows: the tile
// distances as TopkEpi computes them; every column whose distance is at most
// the row's thr is appended to the row's list (coll_n / coll_i, cap entries
// each; the count keeps growing past cap, which tells the reader the list
// overflowed, and a thread stops appending once it sees that).  No tiles at
// all unless the row count exceeds min_rows.
struct ThreshEpi {
    struct Params {
        const int *m_dev;
        int min_rows;
        unsigned nb_tiles;
        size_t n;
        const float *r1, *r2, *c1, *c2;
        const float *thr;
        int *coll_n;
        int *coll_i;
        int cap;
    };
    __device__ static bool slice(const Params &p, int &mb, unsigned &nb0, unsigned &nb1) {
        const int m = *p.m_dev;
        if (m <= p.min_rows) return false;
        const int num_mb = (m + TC_BM - 1) / TC_BM;
        if (num_mb <= 0 || num_mb > (int)gridDim.x) return false;
        const int S = (int)gridDim.x / num_mb;
        if ((int)blockIdx.x >= num_mb * S) return false;
        mb = (int)blockIdx.x / S;
        const int sl = (int)blockIdx.x % S;
        nb0 = (unsigned)(((size_t)p.nb_tiles * sl) / S);
        nb1 = (unsigned)(((size_t)p.nb_tiles * (sl + 1)) / S);
        return true;
    }
    __device__ static int tiles(const Params &p) {
        int mb;
        unsigned nb0, nb1;
        return slice(p, mb, nb0, nb1) ? (int)(nb1 - nb0) : 0;
    }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) {
        unsigned nb0, nb1;
        slice(p, mb, nb0, nb1);
        nb = (int)nb0 + t;
    }
    struct State {
        int rit, m;
        float rr1 = 0.0f, rr2 = 0.0f, T = -INFINITY;
        bool full = false;
        __device__ State(const Params &p, int row_in_tile) : rit(row_in_tile) {
            int mb;
            unsigned nb0, nb1;
            m = *p.m_dev;
            const bool valid = slice(p, mb, nb0, nb1);
            const int row = valid ? mb * TC_BM + rit : 0;
            if (valid && row < m) {
                rr1 = __ldg(p.r1 + row);
                rr2 = __ldg(p.r2 + row);
                T = __ldg(p.thr + row);
            }
        }
        __device__ void tile(const Params &p, int mb, int nb, uint32_t y0, uint32_t) {
            const int row = mb * TC_BM + rit;
            const bool row_ok = row < m;
            const size_t colbase = (size_t)nb * TC_BN;
#pragma unroll 1
            for (int ch = 0; ch < TC_BN / 32; ++ch) {
                float c[32];
                ld_sum32(y0 + 32 * ch, c);  // warp-collective: every lane loads
                if (!row_ok || full) continue;
                const size_t col0 = colbase + ch * 32;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const size_t col = col0 + j;
                    if (col >= p.n) break;
                    const float ipt = __fmul_rn(__fmul_rn(c[j], rr1), __ldg(p.c1 + col));
                    float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + col)), __fmul_rn(2.0f, ipt));
                    d = d > 0.0f ? d : 0.0f;
                    if (d <= T && !full) {
                        const int pos = atomicAdd(p.coll_n + row, 1);
                        if (pos < p.cap)
                            p.coll_i[(size_t)row * p.cap + pos] = (int)col;
                        else
                            full = true;
                    }
                }
            }
        }
        __device__ void finish(const Params &) {}
    };
};

// ---- epilogue policies of tcw_kernel: each thread holds one row's running
// sums of TW_COLS columns (half h of the 256-column tile) in registers.
struct WDist {
    static constexpr bool kDirect = false;  // running sums promoted into registers
    using Params = DistEpi::Params;
    __device__ static int tiles(const Params &p) { return GridTiles::count(p.g.num_tiles); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) { p.g.at(t, mb, nb); }
    struct State {
        int rit, h;
        bool vec;
        __device__ State(const Params &p, int row_in_tile, int half)
            : rit(row_in_tile), h(half),
              vec(((p.ldo & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.out) & 15) == 0)) {}
        // d = max(0, r2 + c2 - 2 (C r1) c1) from the registers
        __device__ void tile(const Params &p, int mb, int nb, const float (&y)[TW_COLS]) {
            const size_t row = (size_t)mb * TC_BM + rit;
            if (row >= p.m) return;
            const float rr1 = __ldg(p.r1 + row), rr2 = __ldg(p.r2 + row);
            float *orow = p.out + row * p.ldo;
            const size_t cbase = (size_t)nb * TW_BN + TW_COLS * h;
#pragma unroll
            for (int g = 0; g < TW_COLS / 4; ++g) {  // groups of 4 columns
                const size_t col0 = cbase + 4 * g;
                if (col0 >= p.n) break;
                float dv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const size_t col = col0 + u < p.n ? col0 + u : p.n - 1;
                    const float ipt = __fmul_rn(__fmul_rn(y[4 * g + u], rr1), __ldg(p.c1 + col));
                    const float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + col)), __fmul_rn(2.0f, ipt));
                    dv[u] = d > 0.0f ? d : 0.0f;
                }
                if (vec && col0 + 4 <= p.n) {
                    *reinterpret_cast<float4 *>(orow + col0) = make_float4(dv[0], dv[1], dv[2], dv[3]);
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (col0 + u < p.n) orow[col0 + u] = dv[u];
                }
            }
        }
        __device__ void finish(const Params &) {}
    };
};

// The top-k over 256-wide column tiles: each thread keeps the best k of its
// half of the columns, so a (row, slice) has two partial lists, written to
// part_d / part_i [((cta * 128 + row) * 2 + half)][kCandMax].  The list lives
// in the thread's local frame and is touched only on an insertion; the
// per-column test reads the k-th entry kept in registers.
struct WTopk {
    static constexpr bool kDirect = false;
    using Params = TopkEpi::Params;  // nb_tiles counts 256-wide tiles
    __device__ static int tiles(const Params &p) { return TopkEpi::tiles(p); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) {
        TopkEpi::tile_at(p, t, mb, nb);
    }
    struct State {
        int rit, h, m;
        bool valid;
        float rr1 = 0.0f, rr2 = 0.0f;
        float bd[kCandMax];
        int bi[kCandMax];
        float thr_d = INFINITY;
        int thr_i = 0x7fffffff;
        __device__ State(const Params &p, int row_in_tile, int half) : rit(row_in_tile), h(half) {
            int mb;
            unsigned nb0, nb1;
            m = *p.m_dev;
            valid = TopkEpi::slice(p, mb, nb0, nb1);
            const int row = valid ? mb * TC_BM + rit : 0;
            if (valid && row < m) {
                rr1 = __ldg(p.r1 + row);
                rr2 = __ldg(p.r2 + row);
            }
#pragma unroll
            for (int t = 0; t < kCandMax; ++t) {
                bd[t] = INFINITY;
                bi[t] = 0x7fffffff;
            }
        }
        __device__ void tile(const Params &p, int mb, int nb, const float (&y)[TW_COLS]) {
            if (mb * TC_BM + rit >= m) return;
            const size_t cbase = (size_t)nb * TW_BN + TW_COLS * h;
            float td = thr_d;
            int ti = thr_i;
#pragma unroll
            for (int j = 0; j < TW_COLS; ++j) {
                const size_t col = cbase + j;
                if (col >= p.n) break;
                const float ipt = __fmul_rn(__fmul_rn(y[j], rr1), __ldg(p.c1 + col));
                float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + col)), __fmul_rn(2.0f, ipt));
                d = d > 0.0f ? d : 0.0f;
                const int ci = (int)col;
                if (better(d, ci, td, ti)) {
                    const TopkEntry e = topk_insert(bd, bi, p.k, d, ci);
                    td = e.d;
                    ti = e.i;
                }
            }
            thr_d = td;
            thr_i = ti;
        }
        __device__ void finish(const Params &p) {
            if (!valid) return;
            int mb;
            unsigned nb0, nb1;
            TopkEpi::slice(p, mb, nb0, nb1);
            if (mb * TC_BM + rit >= m) return;
            const size_t o = (((size_t)blockIdx.x * TC_BM + rit) * 2 + h) * kCandMax;
#pragma unroll
            for (int u = 0; u < kCandMax; ++u)
                if (u < p.k) {
                    p.part_d[o + u] = bd[u];
                    p.part_i[o + u] = bi[u];
                }
        }
    };
};

// The top-k over 256-wide column tiles whose sums run over the whole K in one
// tensor-memory buffer (no promoted chunks; `kDirect`): the epilogue threads
// read their row's 128 columns of the finished tile from tensor memory in
// 16-column pieces and keep a register list of the best kCandMax, as TopkEpi
// does.  Two partial lists per (row, slice), as WTopk.  Without promotion
// the 128 x 256 tile needs no running sums in registers, which is what leaves
// the registers for the list.
struct WTopkD {
    static constexpr bool kDirect = true;
    using Params = TopkEpi::Params;  // nb_tiles counts 256-wide tiles
    __device__ static int tiles(const Params &p) { return TopkEpi::tiles(p); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) {
        TopkEpi::tile_at(p, t, mb, nb);
    }
    struct State {
        int rit, h, m;
        bool valid;
        float rr1 = 0.0f, rr2 = 0.0f;
        float bd[kCandMax];
        int bi[kCandMax];
        __device__ State(const Params &p, int row_in_tile, int half) : rit(row_in_tile), h(half) {
            int mb;
            unsigned nb0, nb1;
            m = *p.m_dev;
            valid = TopkEpi::slice(p, mb, nb0, nb1);
            const int row = valid ? mb * TC_BM + rit : 0;
            if (valid && row < m) {
                rr1 = __ldg(p.r1 + row);
                rr2 = __ldg(p.r2 + row);
            }
#pragma unroll
            for (int t = 0; t < kCandMax; ++t) {
                bd[t] = INFINITY;
                bi[t] = 0x7fffffff;
            }
        }
        // X: this thread's lane and first column of the tile's sums
        // as TopkEpi::State::tile, with the row's published bound (p.gthr)
        __device__ void tile_tmem(const Params &p, int mb, int nb, uint32_t X) {
            const int row = mb * TC_BM + rit;
            const bool row_ok = row < m;
            const size_t cbase = (size_t)nb * TW_BN + TW_COLS * h;
            const unsigned long long g = (row_ok && p.gthr) ? ld_volatile_u64(p.gthr + row) : ~0ull;
#pragma unroll 1
            for (int ch = 0; ch < TW_COLS / 16; ++ch) {
                uint32_t r[16];
                __syncwarp();
                tmem_ld16_nw(X + 16 * ch, r);  // warp-collective: every lane loads
                tmem_wait_ld();
                if (!row_ok) continue;
                const size_t col0 = cbase + ch * 16;
                const unsigned long long own = topk_key(bd[kCandMax - 1], bi[kCandMax - 1]);
                const unsigned long long T = own < g ? own : g;
                float c[16];
                uint32_t pass = 0u;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const size_t col = col0 + j;
                    const size_t cc = col < p.n ? col : p.n - 1;
                    const float ipt = __fmul_rn(__fmul_rn(__uint_as_float(r[j]), rr1), __ldg(p.c1 + cc));
                    float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + cc)), __fmul_rn(2.0f, ipt));
                    d = d > 0.0f ? d : 0.0f;
                    c[j] = d;
                    if (col < p.n && topk_key(d, (int)col) < T) pass |= 1u << j;
                }
                if (pass) {
                    float sd[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) sd[j] = c[j];
                    do {
                        const int j = __ffs(pass) - 1;
                        pass &= pass - 1u;
                        const float d = sd[j];
                        const int ci = (int)(col0 + (size_t)j);
                        const unsigned long long kj = topk_key(d, ci);
                        if (kj < topk_key(bd[kCandMax - 1], bi[kCandMax - 1]) && kj < g)
                            reg_insert(bd, bi, d, ci);
                    } while (pass);
                }
            }
            if (row_ok && p.gthr) {
                const unsigned long long own = topk_key(bd[kCandMax - 1], bi[kCandMax - 1]);
                if (own < g) atomicMin(p.gthr + row, own);
            }
        }
        __device__ void finish(const Params &p) {
            if (!valid) return;
            int mb;
            unsigned nb0, nb1;
            TopkEpi::slice(p, mb, nb0, nb1);
            if (mb * TC_BM + rit >= m) return;
            const size_t o = (((size_t)blockIdx.x * TC_BM + rit) * 2 + h) * kCandMax;
#pragma unroll
            for (int u = 0; u < kCandMax; ++u)
                if (u < p.k) {
                    p.part_d[o + u] = bd[u];
                    p.part_i[o + u] = bi[u];
                }
        }
    };
};

// The threshold collection (as ThreshEpi) over 256-wide column tiles whose
// sums run over the whole K in one tensor-memory buffer, read in place.
struct WThreshD {
    static constexpr bool kDirect = true;
    using Params = ThreshEpi::Params;  // nb_tiles counts 256-wide tiles
    __device__ static int tiles(const Params &p) { return ThreshEpi::tiles(p); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) {
        ThreshEpi::tile_at(p, t, mb, nb);
    }
    struct State {
        int rit, h, m;
        float rr1 = 0.0f, rr2 = 0.0f, T = -INFINITY;
        bool full = false;
        __device__ State(const Params &p, int row_in_tile, int half) : rit(row_in_tile), h(half) {
            int mb;
            unsigned nb0, nb1;
            m = *p.m_dev;
            const bool valid = ThreshEpi::slice(p, mb, nb0, nb1);
            const int row = valid ? mb * TC_BM + rit : 0;
            if (valid && row < m) {
                rr1 = __ldg(p.r1 + row);
                rr2 = __ldg(p.r2 + row);
                T = __ldg(p.thr + row);
            }
        }
        __device__ void tile_tmem(const Params &p, int mb, int nb, uint32_t X) {
            const int row = mb * TC_BM + rit;
            const bool row_ok = row < m;
            const size_t cbase = (size_t)nb * TW_BN + TW_COLS * h;
#pragma unroll 1
            for (int ch = 0; ch < TW_COLS / 16; ++ch) {
                uint32_t r[16];
                __syncwarp();
                tmem_ld16_nw(X + 16 * ch, r);  // warp-collective: every lane loads
                tmem_wait_ld();
                if (!row_ok || full) continue;
                const size_t col0 = cbase + ch * 16;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const size_t col = col0 + j;
                    if (col >= p.n) break;
                    const float ipt = __fmul_rn(__fmul_rn(__uint_as_float(r[j]), rr1), __ldg(p.c1 + col));
                    float d = __fsub_rn(__fadd_rn(rr2, __ldg(p.c2 + col)), __fmul_rn(2.0f, ipt));
                    d = d > 0.0f ? d : 0.0f;
                    if (d <= T && !full) {
                        const int pos = atomicAdd(p.coll_n + row, 1);
                        if (pos < p.cap)
                            p.coll_i[(size_t)row * p.cap + pos] = (int)col;
                        else
                            full = true;
                    }
                }
            }
        }
        __device__ void finish(const Params &) {}
    };
};

// The QJL-corrected symmetric distances (tq_symq.cu): Y0 = C1, Y1 = C2,
// ip_mse = C1 s1a s1b, corr = clamp(C2 s2a s2b, +-|ip_mse|),
// ip = (ip_mse + corr) na nb, d = max(0, na^2 + nb^2 - 2 ip), with the
// per-row scalars s = [s1, norm, s2, ...] (8 floats per row).
struct SymqEpi {
    struct Params {
        GridTiles g;
        size_t m, n;
        const float *sa, *sb;
        float *out;
        size_t ldo;
    };
    __device__ static int tiles(const Params &p) { return GridTiles::count(p.g.num_tiles); }
    __device__ static void tile_at(const Params &p, int t, int &mb, int &nb) { p.g.at(t, mb, nb); }
    struct State {
        int rit;
        bool vec;
        __device__ State(const Params &p, int row_in_tile)
            : rit(row_in_tile),
              vec(((p.ldo & 3) == 0) && ((reinterpret_cast<uintptr_t>(p.out) & 15) == 0)) {}
        __device__ void tile(const Params &p, int mb, int nb, uint32_t y0, uint32_t y1) {
            const size_t row = (size_t)mb * TC_BM + rit;
            const bool row_ok = row < p.m;
            const float s1a = row_ok ? __ldg(p.sa + 8 * row) : 0.0f;
            const float na = row_ok ? __ldg(p.sa + 8 * row + 1) : 0.0f;
            const float s2a = row_ok ? __ldg(p.sa + 8 * row + 2) : 0.0f;
            const float na2 = __fmul_rn(na, na);
            float *orow = p.out + row * p.ldo;
#pragma unroll 1
            for (int ch = 0; ch < TC_BN / 32; ++ch) {
                float c1[32], c2[32];
                ld_sum32(y0 + 32 * ch, c1);
                ld_sum32(y1 + 32 * ch, c2);
                const size_t col0 = (size_t)nb * TC_BN + ch * 32;
                if (!row_ok || col0 >= p.n) continue;
                float dv[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const size_t col = col0 + j < p.n ? col0 + j : p.n - 1;
                    const float s1b = __ldg(p.sb + 8 * col), nb_ = __ldg(p.sb + 8 * col + 1);
                    const float s2b = __ldg(p.sb + 8 * col + 2);
                    const float ip_mse = __fmul_rn(__fmul_rn(c1[j], s1a), s1b);
                    const float lim = fabsf(ip_mse);
                    float corr = __fmul_rn(__fmul_rn(c2[j], s2a), s2b);
                    corr = fmaxf(-lim, fminf(lim, corr));
                    const float ip = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), na), nb_);
                    const float d = __fsub_rn(__fadd_rn(na2, __fmul_rn(nb_, nb_)), __fmul_rn(2.0f, ip));
                    dv[j] = d > 0.0f ? d : 0.0f;
                }
                if (vec && col0 + 32 <= p.n) {
                    float4 *o4 = reinterpret_cast<float4 *>(orow + col0);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        o4[j] = make_float4(dv[4 * j], dv[4 * j + 1], dv[4 * j + 2], dv[4 * j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (col0 + j < p.n) orow[col0 + j] = dv[j];
                }
            }
        }
        __device__ void finish(const Params &) {}
    };
};

// Merge of the per-slice candidates: one warp per query row.  Each lane keeps
// the best kCandMax of its slices' lists in registers (each list ascends, so a
// lane stops reading a list at its first entry that does not beat the lane's
// last), then k rounds of a warp arg-min on (d, index) produce the sorted
// top-k.
__global__ void __launch_bounds__(256) topk_merge_kernel(const int *__restrict__ m_dev, int lists,
                                                         int grid_ctas, const float *__restrict__ part_d,
                                                         const int *__restrict__ part_i, int k,
                                                         float *__restrict__ out_d,
                                                         long long *__restrict__ out_i) {
    const int m = *m_dev;
    const int num_mb = (m + TC_BM - 1) / TC_BM;
    if (num_mb <= 0 || num_mb > grid_ctas) return;
    const int S = grid_ctas / num_mb;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < m; row += gridDim.x * wpb) {
        const int mb = row / TC_BM, rit = row % TC_BM;
        float bd[kCandMax];
        int bi[kCandMax];
#pragma unroll
        for (int t = 0; t < kCandMax; ++t) {
            bd[t] = INFINITY;
            bi[t] = 0x7fffffff;
        }
        for (int sl = lane; sl < S * lists; sl += 32) {
            const size_t cta = (size_t)mb * S + sl / lists;
            const size_t o = ((cta * TC_BM + rit) * lists + sl % lists) * kCandMax;
            for (int u = 0; u < k; ++u) {
                const float cd = part_d[o + u];
                const int cx = part_i[o + u];
                // each list ascends: once an entry does not beat this lane's
                // last kept entry, neither does the rest of the list
                if (!better(cd, cx, bd[kCandMax - 1], bi[kCandMax - 1])) break;
                reg_insert(bd, bi, cd, cx);
            }
        }
        // k rounds: warp arg-min of each lane's current head
        int head = 0;
        for (int u = 0; u < k; ++u) {
            float hd = INFINITY;
            int hx = 0x7fffffff;
#pragma unroll
            for (int v = 0; v < kCandMax; ++v)
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

// FP32 planes (TF32 operands): K x rows, 32-value (128-byte) boxes, 128-byte swizzle.
bool make_map_f32(CUtensorMap *map, const void *base, int K, size_t rows, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 4};
    const cuuint32_t box[2] = {(cuuint32_t)SQ_TBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// CH: K blocks per promoted chunk.
template <bool TF32, int STAGES, int CH, bool SPLIT, class Epi, bool DEC = false>
cudaError_t tcp_launch(const TcMaps &maps, const TcShape &sh, const typename Epi::Params &ep,
                       int *err, unsigned grid, cudaStream_t st, const DecSrc &dec = DecSrc{}) {
    static_assert(CH >= 1, "a chunk holds at least one K block");
    if (SPLIT && sh.nseg != 1) return cudaErrorInvalidValue;  // Y[t & 1] needs the second Y
    const size_t smem = (size_t)STAGES * TC_STAGE_BYTES + TC_BAR_BYTES +
                        (DEC ? TC_DEC_TAB_BYTES + (size_t)dec.cbufs * dec.ctile_bytes : 0) + 1024;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    auto kern = tcp_kernel<TF32, STAGES, CH, SPLIT, Epi, DEC>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, tc_threads(SPLIT, DEC), smem, st>>>(maps, sh, ep, err, dec);
    return cudaGetLastError();
}

template <class W, int CH = 4>
cudaError_t tcw_launch(const TcMaps &maps, const TcShape &sh, const typename W::Params &ep, int *err,
                       unsigned grid, cudaStream_t st) {
    if (sh.nseg != 1) return cudaErrorInvalidValue;
    constexpr int STAGES = 2;
    const size_t smem = (size_t)STAGES * TW_STAGE_BYTES + 256 + 1024;
    auto kern = tcw_kernel<STAGES, CH, W>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, TW_THREADS, smem, st>>>(maps, sh, ep, err);
    return cudaGetLastError();
}

bool aligned16(std::initializer_list<const void *> ps) {
    for (const void *p : ps)
        if (reinterpret_cast<uintptr_t>(p) & 15) return false;
    return true;
}

unsigned sm_grid(size_t tiles) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned)(tiles < (size_t)sms ? tiles : (size_t)sms);
}

// BF16 planes of one K segment: A (K x m_pad), B hi (K x n_pad), B lo (k_lo x n_pad).
bool bf16_maps(TcMaps &mp, TcShape &sh, const void *Ah, const void *Al, size_t m_pad,
               const void *Bh, const void *Bl, size_t n_pad, int K, int k_lo) {
    sh = TcShape{};
    sh.nseg = 1;
    sh.KB[0] = K / TC_BK;
    sh.kbx[0] = k_lo / TC_BK;
    sh.a_exact[0] = 0;
    return make_map(&mp.m[0][0], Ah, K, m_pad, TC_BM) && make_map(&mp.m[0][1], Al, K, m_pad, TC_BM) &&
           make_map(&mp.m[0][2], Bh, K, n_pad, TC_BN) && make_map(&mp.m[0][3], Bl, k_lo, n_pad, TC_BN);
}

}  // namespace

// The serving top-k's tile space: {rows per CTA, codes per tile (the B tile,
// i.e. per pipeline stage), stages, K blocks per promoted chunk}.  Every
// variant keeps 128 query rows per CTA (the UMMA M of cta_group::1); chunks
// stay at <= 8 K blocks, the length the exact stage's error bound assumes.
namespace {
constexpr int kTopkShapes[][4] = {
    {TC_BM, TW_BN, 2, 8},  // 0: tcw_kernel, two lists per (row, slice)
    {TC_BM, TC_BN, 3, 8},  // 1
    {TC_BM, TC_BN, 2, 4},  // 2
    {TC_BM, TC_BN, 3, 4},  // 3
    {TC_BM, TC_BN, 2, 8},  // 4
    {TC_BM, TW_BN, 2, 4},  // 5: tcw_kernel
    {TC_BM, TW_BN, 2, 0},  // 6: tcw_kernel, the whole K in one accumulator (0: no chunks)
};
constexpr int kWholeK = 1 << 16;  // chunk length of variant 6: longer than any K
}  // namespace

int tc_topk_variants() { return (int)(sizeof(kTopkShapes) / sizeof(kTopkShapes[0])); }

// The relative error bound of a variant's tensor pass against the sum of its
// terms' magnitudes.  Per term the split-BF16 representation leaves 3 * 2^-16;
// each K = 16 MMA is taken to add at most 2^-20 of (|accumulator| + sum |p|);
// promotions, the planes' FP32 roundings and the reference's own sums add a
// few 1e-7.  With n MMAs per accumulator (a chunk of ch K blocks: 12 per
// block with a lo plane, 8 without; variant 6: every block of K) the sum is
// 3 * 2^-16 + n * 2^-20 + 5e-7, taken with a factor 1.8 and at least 2.5e-4:
// 2.5e-4 for the 8-block chunks (n = 96), 3.6e-4 for variant 6 at K = 1024,
// K_lo = 512 (n = 160).
float tc_topk_kappa(int variant, int K, int k_lo) {
    const int KB = K / TC_BK, kbx = k_lo / TC_BK;
    int n = 0;
    if (variant >= 0 && variant < tc_topk_variants() && kTopkShapes[variant][3] == 0)
        n = 4 * (3 * kbx + 2 * (KB - kbx));
    else
        n = 4 * 3 * 8;  // the longest chunk of the promoted variants, all with a lo plane
    const float kappa = 1.8f * (3.0f / 65536.0f + (float)n / 1048576.0f + 5e-7f);
    return kappa > 2.5e-4f ? kappa : 2.5e-4f;
}
int tc_topk_lists(int variant) { return kTopkShapes[variant][1] == TW_BN ? 2 : 1; }
bool tc_topk_shape(int variant, int out[4]) {
    if (variant < 0 || variant >= tc_topk_variants()) return false;
    for (int i = 0; i < 4; ++i) out[i] = kTopkShapes[variant][i];
    return true;
}

cudaError_t launch_bounded_wait_selftest(int *err, long long budget_cycles, cudaStream_t st) {
    bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(err, budget_cycles);
    return cudaGetLastError();
}

cudaError_t launch_tc_topk(int variant, const void *Ah, const void *Al, size_t rows_pad,
                           const void *Bh, const void *Bl, size_t n_pad, int K, int k_lo,
                           const int *m_dev, size_t n, const float *r1, const float *r2,
                           const float *c1, const float *c2, int k, float *part_d, int *part_i,
                           unsigned long long *gthr, int *err, int grid, cudaStream_t st) {
    if (k < 1 || k > kCandMax || grid < 1 || variant < 0 || variant >= tc_topk_variants())
        return cudaErrorInvalidValue;
    if (K % TC_BK || k_lo % TC_BK || k_lo <= 0 || k_lo > K || rows_pad % TC_BM || n_pad % TC_BN)
        return cudaErrorInvalidValue;
    if (!aligned16({Ah, Al, Bh, Bl})) return cudaErrorMisalignedAddress;
    alignas(64) TcMaps mp;
    TcShape sh{};
    if (!bf16_maps(mp, sh, Ah, Al, rows_pad, Bh, Bl, n_pad, K, k_lo)) return cudaErrorInvalidValue;
    if (tc_topk_lists(variant) == 2) {
        // 128 x 256 tiles (tcw_kernel), two partial lists per (row, slice)
        if (n_pad % TW_BN) return cudaErrorInvalidValue;
        if (!make_map(&mp.m[0][2], Bh, K, n_pad, TW_BN) || !make_map(&mp.m[0][3], Bl, k_lo, n_pad, TW_BN))
            return cudaErrorInvalidValue;
        const TopkEpi::Params ep{m_dev, (unsigned)(n_pad / TW_BN), n, r1, r2, c1, c2, k, part_d, part_i, gthr};
        if (variant == 6) return tcw_launch<WTopkD, kWholeK>(mp, sh, ep, err, (unsigned)grid, st);
        if (variant == 5) return tcw_launch<WTopk, 4>(mp, sh, ep, err, (unsigned)grid, st);
        return tcw_launch<WTopk, 8>(mp, sh, ep, err, (unsigned)grid, st);
    }
    const TopkEpi::Params ep{m_dev, (unsigned)(n_pad / TC_BN), n, r1, r2, c1, c2, k, part_d, part_i, gthr};
    switch (variant) {
        case 2: return tcp_launch<false, 2, 4, true, TopkEpi>(mp, sh, ep, err, (unsigned)grid, st);
        case 3: return tcp_launch<false, 3, 4, true, TopkEpi>(mp, sh, ep, err, (unsigned)grid, st);
        case 4: return tcp_launch<false, 2, 8, true, TopkEpi>(mp, sh, ep, err, (unsigned)grid, st);
        default: return tcp_launch<false, 3, 8, true, TopkEpi>(mp, sh, ep, err, (unsigned)grid, st);
    }
}

namespace {

// A maps of one K segment for the decoded-B kernels (no B planes).
bool a_maps(TcMaps &mp, TcShape &sh, const void *Ah, const void *Al, size_t m_pad, int K, int kbx) {
    sh = TcShape{};
    sh.nseg = 1;
    sh.KB[0] = K / TC_BK;
    sh.kbx[0] = kbx;
    sh.a_exact[0] = 0;
    return make_map(&mp.m[0][0], Ah, K, m_pad, TC_BM) && make_map(&mp.m[0][1], Al, K, m_pad, TC_BM);
}

bool dec_ok(const DecSrc &d, int K) {
    return d.codes && d.centroids && d.cs % 4 == 0 && (reinterpret_cast<uintptr_t>(d.codes) & 15) == 0 &&
           d.kbc >= 1 && d.kbc <= K / TC_BK && d.levels >= 1 && d.levels <= 256;
}

// Code-tile buffers of a DEC launch with `stages` pipeline stages: two (the
// next tile's copy overlaps this one's decode) when they fit, else one.
DecSrc with_code_buffers(DecSrc d, int stages) {
    d.ctile_bytes = (int)(((size_t)TC_BN * d.cs + 127) & ~size_t(127));
    const size_t fixed = (size_t)stages * TC_STAGE_BYTES + TC_BAR_BYTES + TC_DEC_TAB_BYTES + 1024;
    d.cbufs = fixed + 2 * (size_t)d.ctile_bytes <= 227 * 1024 ? 2
              : fixed + (size_t)d.ctile_bytes <= 227 * 1024 ? 1 : 0;
    return d;
}

}  // namespace

bool tc_topk_dec_ok(int variant, int cs) {
    if (variant < 1 || variant > 4 || cs <= 0) return false;
    DecSrc d;
    d.cs = cs;
    return with_code_buffers(d, (variant == 2 || variant == 4) ? 2 : 3).cbufs > 0;
}

cudaError_t launch_tc_topk_dec(int variant, const void *Ah, const void *Al, size_t rows_pad,
                               const DecSrc &dec, size_t n_pad, int K, const int *m_dev, size_t n,
                               const float *r1, const float *r2, const float *c1, const float *c2,
                               int k, float *part_d, int *part_i, unsigned long long *gthr, int *err,
                               int grid, cudaStream_t st) {
    if (k < 1 || k > kCandMax || grid < 1 || !tc_topk_dec_ok(variant, dec.cs)) return cudaErrorInvalidValue;
    if (K % TC_BK || rows_pad % TC_BM || n_pad % TC_BN || !dec_ok(dec, K) || dec.kbc * 2 != K / TC_BK ||
        !dec.fc || !dec.fs || n > n_pad)
        return cudaErrorInvalidValue;
    if (!aligned16({Ah, Al})) return cudaErrorMisalignedAddress;
    alignas(64) TcMaps mp;
    TcShape sh{};
    if (!a_maps(mp, sh, Ah, Al, rows_pad, K, dec.kbc)) return cudaErrorInvalidValue;
    const TopkEpi::Params ep{m_dev, (unsigned)(n_pad / TC_BN), n, r1, r2, c1, c2, k, part_d, part_i, gthr};
    const int stages = (variant == 2 || variant == 4) ? 2 : 3;
    const DecSrc d = with_code_buffers(dec, stages);
    if (d.cbufs == 0) return cudaErrorInvalidValue;  // the code tile does not fit beside the stages
    switch (variant) {
        case 2: return tcp_launch<false, 2, 4, true, TopkEpi, true>(mp, sh, ep, err, (unsigned)grid, st, d);
        case 3: return tcp_launch<false, 3, 4, true, TopkEpi, true>(mp, sh, ep, err, (unsigned)grid, st, d);
        case 4: return tcp_launch<false, 2, 8, true, TopkEpi, true>(mp, sh, ep, err, (unsigned)grid, st, d);
        default: return tcp_launch<false, 3, 8, true, TopkEpi, true>(mp, sh, ep, err, (unsigned)grid, st, d);
    }
}

cudaError_t launch_tc_thresh(const void *Ah, const void *Al, size_t rows_pad, const void *Bh,
                             const void *Bl, const DecSrc *dec, size_t n_pad, int K, int k_lo,
                             const int *m_dev, int min_rows, size_t n, const float *r1,
                             const float *r2, const float *c1, const float *c2, const float *thr,
                             int *coll_n, int *coll_i, int cap, int *err, int grid, cudaStream_t st) {
    if (grid < 1 || cap < 1 || K % TC_BK || rows_pad % TC_BM || n_pad % TC_BN || n > n_pad)
        return cudaErrorInvalidValue;
    if (!aligned16({Ah, Al})) return cudaErrorMisalignedAddress;
    const ThreshEpi::Params ep{m_dev, min_rows, (unsigned)(n_pad / TC_BN), n,      r1,  r2,
                               c1,    c2,       thr,                      coll_n, coll_i, cap};
    alignas(64) TcMaps mp;
    TcShape sh{};
    if (dec) {
        // variant 4's shape with decoded B tiles
        if (!dec_ok(*dec, K) || dec->kbc * 2 != K / TC_BK || !dec->fc || !dec->fs)
            return cudaErrorInvalidValue;
        if (!a_maps(mp, sh, Ah, Al, rows_pad, K, dec->kbc)) return cudaErrorInvalidValue;
        const DecSrc d = with_code_buffers(*dec, 2);
        if (d.cbufs == 0) return cudaErrorInvalidValue;
        return tcp_launch<false, 2, 8, true, ThreshEpi, true>(mp, sh, ep, err, (unsigned)grid, st, d);
    }
    if (k_lo % TC_BK || k_lo <= 0 || k_lo > K) return cudaErrorInvalidValue;
    if (!aligned16({Bh, Bl})) return cudaErrorMisalignedAddress;
    if (!bf16_maps(mp, sh, Ah, Al, rows_pad, Bh, Bl, n_pad, K, k_lo)) return cudaErrorInvalidValue;
    if (n_pad % TW_BN == 0) {
        // variant 6's shape: 128 x 256 tiles, the whole K in one accumulator
        if (!make_map(&mp.m[0][2], Bh, K, n_pad, TW_BN) || !make_map(&mp.m[0][3], Bl, k_lo, n_pad, TW_BN))
            return cudaErrorInvalidValue;
        ThreshEpi::Params ew = ep;
        ew.nb_tiles = (unsigned)(n_pad / TW_BN);
        return tcw_launch<WThreshD, kWholeK>(mp, sh, ew, err, (unsigned)grid, st);
    }
    return tcp_launch<false, 2, 8, true, ThreshEpi>(mp, sh, ep, err, (unsigned)grid, st);
}

int tc_thresh_variant(bool decoded, size_t n_pad) { return (!decoded && n_pad % TW_BN == 0) ? 6 : 4; }

cudaError_t launch_topk_merge(const int *m_dev, int grid_ctas, int lists, const float *part_d,
                              const int *part_i, int k, size_t max_rows, float *out_d,
                              long long *out_i, cudaStream_t st) {
    if (lists < 1 || lists > 2) return cudaErrorInvalidValue;
    const int wpb = 8;
    const unsigned blocks = (unsigned)((max_rows + wpb - 1) / wpb);
    topk_merge_kernel<<<blocks ? blocks : 1, 32 * wpb, 0, st>>>(m_dev, lists, grid_ctas, part_d,
                                                                part_i, k, out_d, out_i);
    return cudaGetLastError();
}

cudaError_t launch_tc_dist(const void *Ah, const void *Al, const void *Bh, const void *Bl, int K,
                           int k_lo, size_t m, size_t m_pad, size_t n, size_t n_pad,
                           const float *r1, const float *r2, const float *c1, const float *c2,
                           float *out, size_t ldo, int *err, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    if (K % TC_BK || k_lo % TC_BK || k_lo <= 0 || k_lo > K || m_pad % TC_BM || n_pad % TC_BN ||
        m > m_pad || n > n_pad)
        return cudaErrorInvalidValue;
    if (!aligned16({Ah, Al, Bh, Bl})) return cudaErrorMisalignedAddress;
    alignas(64) TcMaps mp;
    TcShape sh{};
    if (!bf16_maps(mp, sh, Ah, Al, m_pad, Bh, Bl, n_pad, K, k_lo)) return cudaErrorInvalidValue;
    const unsigned num_mb = (unsigned)(m_pad / TC_BM);
    const size_t tiles = (size_t)num_mb * (n_pad / TC_BN);
    if (tiles > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    if (n_pad % TW_BN == 0) {
        // 128 x 256 tiles (tcw_kernel): B maps with 256-row boxes
        if (!make_map(&mp.m[0][2], Bh, K, n_pad, TW_BN) || !make_map(&mp.m[0][3], Bl, k_lo, n_pad, TW_BN))
            return cudaErrorInvalidValue;
        const size_t wtiles = (size_t)num_mb * (n_pad / TW_BN);
        const DistEpi::Params ep{GridTiles{num_mb, (unsigned)wtiles}, m, n, r1, r2, c1, c2, out, ldo};
        // Chunk length: asymmetric planes (B lo narrower than K: a query against
        // codes) take 8 K blocks per chunk; symmetric planes, whose code-against-
        // itself terms are squares of centroid values, 4 (their drift per chunk
        // is larger against a BF16-pair floor of 5-7e-6).
        if (k_lo < K) return tcw_launch<WDist, 8>(mp, sh, ep, err, sm_grid(wtiles), st);
        return tcw_launch<WDist, 4>(mp, sh, ep, err, sm_grid(wtiles), st);
    }
    const DistEpi::Params ep{GridTiles{num_mb, (unsigned)tiles}, m, n, r1, r2, c1, c2, out, ldo};
    return tcp_launch<false, 3, 4, true, DistEpi>(mp, sh, ep, err, sm_grid(tiles), st);
}

bool tc_dist_dec_fits(int cs) {
    DecSrc d;
    d.cs = cs;
    return cs > 0 && with_code_buffers(d, 2).cbufs > 0;
}

cudaError_t launch_tc_dist_dec(const void *Ah, const void *Al, size_t m, size_t m_pad, const DecSrc &dec,
                               size_t n_pad, int K, const float *r1, const float *r2, const float *c1,
                               const float *c2, float *out, size_t ldo, int *err, cudaStream_t st) {
    if (m == 0 || dec.n == 0) return cudaSuccess;
    const bool sym = dec.fc == nullptr;
    if (K % TC_BK || m_pad % TC_BM || n_pad % TC_BN || m > m_pad || dec.n > n_pad || !dec_ok(dec, K))
        return cudaErrorInvalidValue;
    // symmetric: the whole K is centroid values; asymmetric: centroid half + sign half
    if (sym ? dec.kbc != K / TC_BK : (dec.kbc * 2 != K / TC_BK || !dec.fs)) return cudaErrorInvalidValue;
    if (!aligned16({Ah, Al})) return cudaErrorMisalignedAddress;
    alignas(64) TcMaps mp;
    TcShape sh{};
    if (!a_maps(mp, sh, Ah, Al, m_pad, K, dec.kbc)) return cudaErrorInvalidValue;
    const unsigned num_mb = (unsigned)(m_pad / TC_BM);
    const size_t tiles = (size_t)num_mb * (n_pad / TC_BN);
    if (tiles > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    const DecSrc d = with_code_buffers(dec, 2);
    if (d.cbufs == 0) return cudaErrorInvalidValue;  // the code tile does not fit beside the stages
    const DistEpi::Params ep{GridTiles{num_mb, (unsigned)tiles}, m, dec.n, r1, r2, c1, c2, out, ldo};
    // chunk lengths as the planes kernels: 8 K blocks asymmetric, 4 symmetric
    if (sym) return tcp_launch<false, 2, 4, true, DistEpi, true>(mp, sh, ep, err, sm_grid(tiles), st, d);
    return tcp_launch<false, 2, 8, true, DistEpi, true>(mp, sh, ep, err, sm_grid(tiles), st, d);
}

cudaError_t launch_tc_symq(const void *A1h, const void *A1l, const void *B1h, const void *B1l,
                           int K1, const void *A2h, const void *A2l, const void *B2h,
                           const void *B2l, int K2, bool exact2, size_t m, size_t m_pad, size_t n,
                           size_t n_pad, const float *sa, const float *sb, float *out, size_t ldo,
                           int *err, cudaStream_t st) {
    if (m == 0 || n == 0) return cudaSuccess;
    if (K1 <= 0 || K2 <= 0 || K1 % SQ_TBK || K2 % SQ_TBK || m_pad % TC_BM || n_pad % TC_BN ||
        m > m_pad || n > n_pad)
        return cudaErrorInvalidValue;
    if (!aligned16({A1h, A1l, B1h, B1l, A2h, A2l, B2h, B2l})) return cudaErrorMisalignedAddress;
    alignas(64) TcMaps mp;
    const void *pl[2][4] = {{A1h, A1l, B1h, B1l}, {A2h, A2l, B2h, B2l}};
    const int Ks[2] = {K1, K2};
    for (int sg = 0; sg < 2; ++sg)
        for (int o = 0; o < 4; ++o)
            if (!make_map_f32(&mp.m[sg][o], pl[sg][o], Ks[sg], o < 2 ? m_pad : n_pad, o < 2 ? TC_BM : TC_BN))
                return cudaErrorInvalidValue;
    TcShape sh{};
    sh.nseg = 2;
    sh.KB[0] = K1 / SQ_TBK;
    sh.KB[1] = K2 / SQ_TBK;
    sh.kbx[0] = sh.KB[0];
    sh.kbx[1] = exact2 ? 0 : sh.KB[1];
    sh.a_exact[0] = 0;
    sh.a_exact[1] = exact2 ? 1 : 0;
    sh.whole[1] = exact2 ? 1 : 0;
    const unsigned num_mb = (unsigned)(m_pad / TC_BM);
    const size_t tiles = (size_t)num_mb * (n_pad / TC_BN);
    if (tiles > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    const SymqEpi::Params ep{GridTiles{num_mb, (unsigned)tiles}, m, n, sa, sb, out, ldo};
    return tcp_launch<true, 3, 4, false, SymqEpi>(mp, sh, ep, err, sm_grid(tiles), st);
}

}  // namespace tq
