// tq_kernels.cu -- sm_100a kernels of the TurboQuant encode-and-scan path.
//
//   encode_kernel   fused encodeVector (space_turbo_quant.h:339-396): norm,
//                   sign flip + FWHT, sigma, Lloyd-Max quantize, residual,
//                   gamma, QJL sign flip + FWHT, pack + trailer.  Bit-exact
//                   with the reference's pinned Release build.
//   prepare_kernel  prepareQuery (:439-460).
//   scan_kernel     asymmetric distSearch* (:659-686, 951-983) over a code
//                   stream (distanceBatch1ToN/MToN :577-599) and the MSE-only
//                   symmetric distBuild* (:688-714, 985-1019) (MToNSymmetric
//                   :602-615).
//
// Rounding discipline: every float operation whose rounding the reference
// fixes is written with an explicit round-to-nearest intrinsic (__fadd_rn,
// __fmul_rn, __fmaf_rn, __fdiv_rn, __fsqrt_rn) so that nvcc cannot contract
// or reassociate it.
#include "tq_async.cuh"
#include "tq_internal.h"
#include "tq_rht.cuh"

#include <cstdint>

namespace tq {
namespace {

// Per-warp shared bytes of the encode kernel: vpw vectors of D+8 floats, vpw x D
// quantizer indices, vpw staged codes.
__host__ __device__ __forceinline__ int encode_warp_bytes(int D, int cs, int vpw) {
    return vpw * 4 * (D + 8) + vpw * D + align16(vpw * cs);
}

// ---------------------------------------------------------------------------
// Quantizer of CH values held in registers (quantize, space_turbo_quant.h:
// 332-337), each replaced by its residual x - c[idx] * sigma as one FMA
// (:366); emit(t, idx) receives the indices.  The table loads of the CH values
// are independent of one another, so they overlap.
//   kQuantBucket: the bucket table when every bucket holds at most one
//                 boundary (qlut_k = 1: b = 6..9), idx = lo + (z > B[lo]);
//   kQuantRegs:   nb <= 15 boundaries (b = 2..5) held in registers, padded
//                 with +inf: idx = #{j : z > B[j]} with no table load;
//   kQuantTable:  anything else, through quantize().
// ---------------------------------------------------------------------------
enum { kQuantBucket = 1, kQuantRegs = 2, kQuantTable = 3 };

__device__ __forceinline__ int quant_mode(const Params &P) {
    if (P.lutq) return P.qlut_k == 1 ? kQuantBucket : kQuantTable;
    return P.nb <= 15 ? kQuantRegs : kQuantTable;
}

__device__ __forceinline__ void load_bound_regs(float (&breg)[15], const Params &P,
                                                const float *s_bnd) {
#pragma unroll
    for (int j = 0; j < 15; ++j) breg[j] = (j < P.nb) ? s_bnd[j] : __int_as_float(0x7f800000);
}

template <int NB, int CH, class Emit>
__device__ __forceinline__ void quantize_regs_nb(float (&xr)[CH], float isg, float sg,
                                                 const float (&breg)[15], const float *s_cent,
                                                 Emit emit) {
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const float z = __fmul_rn(xr[t], isg);
        int idx = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j) idx += (z > breg[j]) ? 1 : 0;
        xr[t] = __fmaf_rn(-s_cent[idx], sg, xr[t]);
        emit(t, idx);
    }
}

template <int CH, class Emit>
__device__ __forceinline__ void quantize_regs(float (&xr)[CH], float isg, float sg, int mode,
                                              const Params &P, const float (&breg)[15],
                                              const float *s_bnd, const uint8_t *s_qlut,
                                              const float *s_cent, Emit emit) {
    if (mode == kQuantBucket) {
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const float z = __fmul_rn(xr[t], isg);
            float y = __fmaf_rn(z, P.qlut_s, P.qlut_c);
            y = fminf(fmaxf(y, 0.0f), (float)(kQlutBuckets - 1));
            int idx = s_qlut[(int)y];
            idx = (idx + ((z > s_bnd[idx]) ? 1 : 0)) & 0xFF;
            xr[t] = __fmaf_rn(-s_cent[idx], sg, xr[t]);
            emit(t, idx);
        }
    } else if (mode == kQuantRegs) {
        // nb = 2^(b-1) - 1: one compare per boundary, the count fixed at compile time
        switch (P.nb) {
            case 1: quantize_regs_nb<1, CH>(xr, isg, sg, breg, s_cent, emit); break;
            case 3: quantize_regs_nb<3, CH>(xr, isg, sg, breg, s_cent, emit); break;
            case 7: quantize_regs_nb<7, CH>(xr, isg, sg, breg, s_cent, emit); break;
            default: quantize_regs_nb<15, CH>(xr, isg, sg, breg, s_cent, emit); break;
        }
    } else {
#pragma unroll
        for (int t = 0; t < CH; ++t) {
            const int idx = quantize(__fmul_rn(xr[t], isg), P, s_bnd, s_qlut);
            xr[t] = __fmaf_rn(-s_cent[idx], sg, xr[t]);
            emit(t, idx);
        }
    }
}

// The bucket quantizer (kQuantBucket) with the flagged bucket table of
// P.qflag and a lane-replicated centroid table: entry e of bucket y is
// lo | 0x80 when a boundary lies inside the bucket, and only then is z
// compared with B[lo] (about 4% of the values at b = 8); crow = table + lane,
// entry idx at crow[32 idx], so the centroid loads of a warp hit 32 distinct
// banks.  Same indices and residuals as quantize_regs.
template <int CH, class Emit>
__device__ __forceinline__ void quantize_regs_flag(float (&xr)[CH], float isg, float sg,
                                                   const Params &P, const float *s_bnd,
                                                   const uint8_t *s_qlutf, const float *crow,
                                                   Emit emit) {
#pragma unroll
    for (int t = 0; t < CH; ++t) {
        const float z = __fmul_rn(xr[t], isg);
        float y = __fmaf_rn(z, P.qlut_s, P.qlut_c);
        y = fminf(fmaxf(y, 0.0f), (float)(kQlutBuckets - 1));
        const int e = s_qlutf[(int)y];
        int idx = e & 0x7F;
        if (e & 0x80) idx += (z > s_bnd[idx]) ? 1 : 0;
        xr[t] = __fmaf_rn(-crow[32 * idx], sg, xr[t]);
        emit(t, idx);
    }
}

// Bytes of encode2's lane-replicated centroid table (P.qflag): levels x 32 floats.
__host__ __device__ __forceinline__ int crep_bytes(const Params &P) { return P.qflag ? P.levels * 128 : 0; }

// ---------------------------------------------------------------------------
// encode: one warp per group of VPW consecutive rows (VPW = 4, or 2 at large
// D, where four vector buffers per warp would leave room for only 4 warps per
// SM).  The reduction chains run on 8 lanes per vector; with VPW = 2 the lane
// groups 2 and 3 repeat the chains of vectors 0 and 1.
// ---------------------------------------------------------------------------
template <int LOG_D, int VPW>
__global__ void __launch_bounds__(256) encode_kernel(const float *__restrict__ X, size_t n,
                                                     uint8_t *__restrict__ out, Params P,
                                                     DevTables T) {
    constexpr int D = 1 << LOG_D;
    constexpr int VS = D + 8;
    extern __shared__ __align__(16) unsigned char smem[];
    load_tables(smem, P, T, true);
    __syncthreads();
    const float *s_cent = reinterpret_cast<const float *>(smem + kTabCentOff);
    const float *s_bnd = reinterpret_cast<const float *>(smem + kTabBndOff);
    const uint32_t *s_rot = reinterpret_cast<const uint32_t *>(smem + kTabRotOff);
    const uint32_t *s_qjl = reinterpret_cast<const uint32_t *>(smem + kTabQjlOff);
    const uint8_t *s_qlut = smem + kTabQlutOff;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int cs = P.cs;
    unsigned char *wbase = smem + kTabBytes + warp * encode_warp_bytes(D, cs, VPW);
    float *buf = reinterpret_cast<float *>(wbase);
    uint8_t *idxb = wbase + VPW * 4 * VS;
    uint8_t *stage = idxb + VPW * D;
    const int g = lane >> 3;
    float *gbuf = buf + (g % VPW) * VS;
    const bool vec4 = ((P.dim & 3) == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const size_t ngroups = (n + VPW - 1) / VPW;

    for (size_t qd = (size_t)blockIdx.x * nwarps + warp; qd < ngroups;
         qd += (size_t)gridDim.x * nwarps) {
        const size_t row0 = qd * VPW;
        const int nv = (n - row0 < (size_t)VPW) ? (int)(n - row0) : VPW;

        // A: rows -> shared memory, zero padded to D (space_turbo_quant.h:347-350)
#pragma unroll
        for (int v = 0; v < VPW; ++v) {
            float *b = buf + v * VS;
            if (v < nv) {
                const float *src = X + (row0 + v) * (size_t)P.dim;
                if (vec4) {
                    const float4 *s4 = reinterpret_cast<const float4 *>(src);
                    for (int i4 = lane; i4 < (P.dim >> 2); i4 += 32) {
                        const float4 x = __ldcs(s4 + i4);
                        const int e = i4 << 2;
                        b[swz(e)] = x.x;
                        b[swz(e + 1)] = x.y;
                        b[swz(e + 2)] = x.z;
                        b[swz(e + 3)] = x.w;
                    }
                } else {
                    for (int i = lane; i < P.dim; i += 32) b[swz(i)] = __ldcs(src + i);
                }
                for (int i = P.dim + lane; i < D; i += 32) b[swz(i)] = 0.0f;
            } else {
                for (int i = lane; i < D; i += 32) b[swz(i)] = 0.0f;
            }
        }
        __syncwarp();

        // B: norm (:342-348)
        const float nsq = chain_sq_reduce(gbuf, P.dim, lane);
        const float norm = __fsqrt_rn(nsq);
        const float inv_norm = (nsq > f32_bits(kNormSqFloorBits)) ? __fdiv_rn(1.0f, norm) : 0.0f;

        // C: rotated = RHT_rot(raw * inv_norm) (:349-351)
#pragma unroll 1
        for (int v = 0; v < VPW; ++v) {
            const float inv = __shfl_sync(kFull, inv_norm, 8 * v);
            fwht_from<LOG_D, 0, true>(buf + v * VS, lane, inv, s_rot, P.wht_scale);
        }

        // D: sigma (:353-359)
        const float var = chain_sq_reduce(gbuf, D, lane);
        float sigma = __fsqrt_rn(__fdiv_rn(var, (float)D));
        float inv_sigma;
        if (f32_bits(kSigmaFloorBits) > sigma) {
            sigma = f32_bits(kSigmaFloorBits);
            inv_sigma = f32_bits(kInvSigmaFloorBits);
        } else {
            inv_sigma = __fdiv_rn(1.0f, sigma);
        }

        // E: quantize + residual (:361-367); the residual is one FMA.  The
        // values are loaded in runs of CH per lane, quantized in registers and
        // stored afterwards (a store between two loads of the buffer would
        // order every element's table loads after the previous element's).
        const int qmode = quant_mode(P);
        float breg[15];
        load_bound_regs(breg, P, s_bnd);
#pragma unroll 1
        for (int v = 0; v < VPW; ++v) {
            const float sg = __shfl_sync(kFull, sigma, 8 * v);
            const float isg = __shfl_sync(kFull, inv_sigma, 8 * v);
            float *b = buf + v * VS;
            uint8_t *ib = idxb + v * D;
            if constexpr (D >= 32) {
                constexpr int PER = D / 32, CH = PER < 16 ? PER : 16;
#pragma unroll 1
                for (int c0 = 0; c0 < PER; c0 += CH) {
                    float xr[CH];
#pragma unroll
                    for (int t = 0; t < CH; ++t) xr[t] = b[swz(lane + 32 * (c0 + t))];
                    quantize_regs<CH>(xr, isg, sg, qmode, P, breg, s_bnd, s_qlut, s_cent,
                                      [&](int t, int idx) { ib[lane + 32 * (c0 + t)] = (uint8_t)idx; });
#pragma unroll
                    for (int t = 0; t < CH; ++t) b[swz(lane + 32 * (c0 + t))] = xr[t];
                }
            } else {
                for (int i = lane; i < D; i += 32) {
                    const int p = swz(i);
                    const float x = b[p];
                    const int idx = quantize(__fmul_rn(x, isg), P, s_bnd, s_qlut);
                    b[p] = __fmaf_rn(-s_cent[idx], sg, x);
                    ib[i] = (uint8_t)idx;
                }
            }
        }
        __syncwarp();

        // F: gamma (:369-372)
        const float gamma = __fsqrt_rn(chain_sq_reduce(gbuf, D, lane));

        // G: RHT_qjl(residual) (:374)
#pragma unroll 1
        for (int v = 0; v < VPW; ++v) fwht_from<LOG_D, 0, false>(buf + v * VS, lane, 1.0f, s_qjl, P.wht_scale);

        // H: pack units + trailer into the staging area (:375-395)
        for (int v = 0; v < nv; ++v) {
            const float *b = buf + v * VS;
            const uint8_t *ib = idxb + v * D;
            uint8_t *st = stage + v * cs;
            if (P.nibble) {
                for (int j = lane; j < P.pb; j += 32) {
                    const unsigned u0 = ((unsigned)ib[2 * j] << 1) | (b[swz(2 * j)] >= 0.0f ? 1u : 0u);
                    const unsigned u1 =
                        ((unsigned)ib[2 * j + 1] << 1) | (b[swz(2 * j + 1)] >= 0.0f ? 1u : 0u);
                    st[j] = (uint8_t)((u0 | (u1 << 4)) & 0xFFu);
                }
            } else {
                for (int i = lane; i < D; i += 32)
                    st[i] = (uint8_t)((((unsigned)ib[i] << 1) | (b[swz(i)] >= 0.0f ? 1u : 0u)) & 0xFFu);
            }
        }
        if ((lane & 7) == 0 && g < nv) {
            uint8_t *t = stage + g * cs + P.pb;
            const uint32_t w[3] = {__float_as_uint(norm), __float_as_uint(gamma), __float_as_uint(sigma)};
#pragma unroll
            for (int q = 0; q < 12; ++q) t[q] = (uint8_t)(w[q >> 2] >> (8 * (q & 3)));
        }
        __syncwarp();

        // I: staged codes -> global (one contiguous run of nv * cs bytes)
        uint8_t *dst = out + row0 * (size_t)cs;
        const int len = nv * cs;
        if (((reinterpret_cast<uintptr_t>(dst) & 15) == 0) && ((len & 15) == 0)) {
            const uint4 *s4 = reinterpret_cast<const uint4 *>(stage);
            uint4 *d4 = reinterpret_cast<uint4 *>(dst);
            for (int i = lane; i < (len >> 4); i += 32) __stcs(d4 + i, s4[i]);
        } else if (((reinterpret_cast<uintptr_t>(dst) & 3) == 0) && ((len & 3) == 0)) {
            const uint32_t *s1 = reinterpret_cast<const uint32_t *>(stage);
            uint32_t *d1 = reinterpret_cast<uint32_t *>(dst);
            for (int i = lane; i < (len >> 2); i += 32) d1[i] = s1[i];
        } else {
            for (int i = lane; i < len; i += 32) dst[i] = stage[i];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// encode2: the same computation for D = 256, 512, 1024 (E = D/32 = 8, 16, 32
// values per lane) with the FWHT held in registers.
//   layout A: lane l holds elements l*E + t; stages 0..log2(E)-1 in registers,
//             stages log2(E)..4 (E < 32) with lane shuffles;
//   one shared-memory transpose;
//   layout B: lane l holds elements 32 t + l; stages 5.. in registers.
// Butterflies of register stride >= 2 use packed FP32x2 add/sub: each half is
// an independent IEEE add or subtract, so every stage output is still the
// single rounding of a + b or a - b and the stage order is unchanged.
// The vector buffer is row-padded (PadLayout below): the float4 layout-A
// accesses, the layout-B accesses and the 8-lane reduction chains are free of
// bank conflicts without per-access index arithmetic.
// ---------------------------------------------------------------------------
typedef unsigned long long u64;

__device__ __forceinline__ u64 fadd2(u64 a, u64 b) {
    u64 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 fsub2(u64 a, u64 b) {
    u64 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 fmul2(u64 a, u64 b) {
    u64 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 mk2(float lo, float hi) {
    u64 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void un2(u64 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// Vector buffer layout of encode2: element e at e + 4 (e >> 5), i.e. every
// 32-float row is followed by 4 floats of padding.  The layout-A float4
// accesses (lane l: elements E l .. E l + E - 1), the layout-B accesses
// (lane l: elements 32 t + l) and the 8-lane reduction chains are all free of
// bank conflicts, and with the unrolled indices every address is a per-lane
// base plus an immediate offset.  VecRow<D> floats per vector (a multiple of
// 32 plus 8, so that the 4 vectors of a warp start 8 banks apart).
template <int E>
struct PadLayout {
    // physical float offset of element e
    __device__ static __forceinline__ int elem(int e) { return e + ((e >> 5) << 2); }
    // physical float offset of chunk c (elements 4c .. 4c + 3)
    __device__ static __forceinline__ int chunk(int c) { return (c << 2) + ((c >> 3) << 2); }
};

template <int D>
__host__ __device__ constexpr int vec_row_floats() {
    return D + D / 8 + 8;
}

// The reference's sum-of-squares tree (as chain_sq_reduce) on a PadLayout
// buffer.  FULL: n = D (a multiple of 32), so there are no leftovers.  Chain k
// (lane k of the 8-lane group) reads elements k + 8 m: four per 32-float row.
template <int E, bool FULL>
__device__ __forceinline__ float chain_sq_reduce2(const float *buf, int n, int lane) {
    if constexpr (FULL) n = 32 * E;
    const int k = lane & 7;
    const int steps = (n & ~7) >> 3;
    float acc = 0.0f;
    int m = 0;
    // 16 steps (4 rows) per iteration: the loads run ahead of the chain
#pragma unroll 1
    for (; m + 16 <= steps; m += 16) {
        const float *base = buf + (m >> 2) * 36 + k;
        float xs[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) xs[i] = base[(i >> 2) * 36 + 8 * (i & 3)];
#pragma unroll
        for (int i = 0; i < 16; ++i) acc = __fadd_rn(acc, __fmul_rn(xs[i], xs[i]));
    }
#pragma unroll 1
    for (; m + 4 <= steps; m += 4) {
        const float *base = buf + (m >> 2) * 36 + k;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float x = base[8 * i];
            acc = __fadd_rn(acc, __fmul_rn(x, x));
        }
    }
    if constexpr (!FULL) {
#pragma unroll 1
        for (; m < steps; ++m) {
            const float x = buf[PadLayout<E>::elem(k + 8 * m)];
            acc = __fadd_rn(acc, __fmul_rn(x, x));
        }
    }
    const float hi = __shfl_down_sync(kFull, acc, 4, 8);
    const float t = __fadd_rn(acc, hi);
    float t0 = __shfl_sync(kFull, t, 0, 8);
    float t1 = __shfl_sync(kFull, t, 1, 8);
    float t2 = __shfl_sync(kFull, t, 2, 8);
    float t3 = __shfl_sync(kFull, t, 3, 8);
    float s = __fadd_rn(__fadd_rn(t0, t2), __fadd_rn(t1, t3));
    if constexpr (FULL) return s;
    int b = n & ~7, r = n - b;
    if (r >= 4) {
        const float x0 = buf[PadLayout<E>::elem(b)], x1 = buf[PadLayout<E>::elem(b + 1)];
        const float x2 = buf[PadLayout<E>::elem(b + 2)], x3 = buf[PadLayout<E>::elem(b + 3)];
        t0 = __fmaf_rn(x0, x0, t0);
        t1 = __fmaf_rn(x1, x1, t1);
        t2 = __fmaf_rn(x2, x2, t2);
        t3 = __fmaf_rn(x3, x3, t3);
        s = __fadd_rn(__fadd_rn(t0, t2), __fadd_rn(t1, t3));
        b += 4;
        r -= 4;
    }
    for (int j = 0; j < r; ++j) {
        const float x = buf[PadLayout<E>::elem(b + j)];
        s = __fmaf_rn(x, x, s);
    }
    return s;
}

// In-register butterfly stage of register stride 2^SREG over E values held as
// E/2 pairs (p[i] = values 2i, 2i+1).
template <int E, int SREG>
__device__ __forceinline__ void reg_stage(u64 (&p)[E / 2]) {
    if constexpr (SREG == 0) {
#pragma unroll
        for (int i = 0; i < E / 2; ++i) {
            float a, b;
            un2(p[i], a, b);
            p[i] = mk2(__fadd_rn(a, b), __fsub_rn(a, b));
        }
    } else {
        constexpr int PS = 1 << (SREG - 1);
#pragma unroll
        for (int i = 0; i < E / 2; ++i) {
            if (!(i & PS)) {
                const u64 a = p[i], b = p[i + PS];
                p[i] = fadd2(a, b);
                p[i + PS] = fsub2(a, b);
            }
        }
    }
}

template <int E, int SREG = 0>
__device__ __forceinline__ void reg_stages(u64 (&p)[E / 2]) {
    if constexpr ((1 << SREG) < E) {
        reg_stage<E, SREG>(p);
        reg_stages<E, SREG + 1>(p);
    }
}

// Cross-lane stages of layout A (element bits log2(E)..4 are lane bits).
template <int E, int LB = 0>
__device__ __forceinline__ void lane_stages(u64 (&p)[E / 2], int lane) {
    constexpr int LE = (E >= 32) ? 5 : (E == 16 ? 4 : 3);
    if constexpr (LE + LB < 5) {
        const int mask = 1 << LB;
        const bool high = lane & mask;
#pragma unroll
        for (int i = 0; i < E / 2; ++i) {
            const u64 y = __shfl_xor_sync(kFull, p[i], mask);
            const u64 x = high ? (p[i] ^ 0x8000000080000000ull) : p[i];
            p[i] = fadd2(y, x);  // low lane: y + x; high lane: y - x (= low - high)
        }
        lane_stages<E, LB + 1>(p, lane);
    }
}

// RHT of one vector held in `buf` (PadLayout<E>): optional pre-multiply, sign flip
// from `sbits` (bit t: element lane*E + t is +1), FWHT, post-multiply.  The
// result is left in layout B in `out` (E values: element 32 t + lane).
template <int E, bool PREMUL>
__device__ __forceinline__ void rht2(float *buf, int lane, float pre, uint32_t sbits, float post,
                                     float (&out)[E]) {
    u64 p[E / 2];
#pragma unroll
    for (int k = 0; k < E / 4; ++k) {
        const float4 x = *reinterpret_cast<const float4 *>(buf + PadLayout<E>::chunk(lane * (E / 4) + k));
        p[2 * k] = mk2(x.x, x.y);
        p[2 * k + 1] = mk2(x.z, x.w);
    }
    const u64 pre2 = mk2(pre, pre);
#pragma unroll
    for (int i = 0; i < E / 2; ++i) {
        if constexpr (PREMUL) p[i] = fmul2(p[i], pre2);
        const u64 flip = ((u64)((~sbits >> (2 * i)) & 1u) << 31) | ((u64)((~sbits >> (2 * i + 1)) & 1u) << 63);
        p[i] ^= flip;
    }
    reg_stages<E>(p);
    lane_stages<E>(p, lane);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < E / 4; ++k) {
        float a, b, c, d;
        un2(p[2 * k], a, b);
        un2(p[2 * k + 1], c, d);
        *reinterpret_cast<float4 *>(buf + PadLayout<E>::chunk(lane * (E / 4) + k)) = make_float4(a, b, c, d);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < E / 2; ++i)
        p[i] = mk2(buf[PadLayout<E>::elem(32 * (2 * i) + lane)], buf[PadLayout<E>::elem(32 * (2 * i + 1) + lane)]);
    reg_stages<E>(p);
    const u64 post2 = mk2(post, post);
#pragma unroll
    for (int i = 0; i < E / 2; ++i) {
        p[i] = fmul2(p[i], post2);
        un2(p[i], out[2 * i], out[2 * i + 1]);
    }
    __syncwarp();
}

// Rows per warp and warps per CTA of encode2.  Byte codes at D = 1024 (168
// registers) run 3 rows per warp in one CTA of 12 warps per SM, three warps
// per scheduler to hide the serial reduction chains; shared memory holds 8
// warps of 4 rows.  Everything else: 4 rows per warp, CTAs of 4 warps.
template <int LOG_D, bool NIBBLE>
__host__ __device__ constexpr int enc2_rpw() { return (LOG_D == 10 && !NIBBLE) ? 3 : 4; }
template <int LOG_D, bool NIBBLE>
__host__ __device__ constexpr int enc2_max_warps() { return (LOG_D == 10 && !NIBBLE) ? 12 : 4; }

// Per-warp shared bytes of encode2: RPW padded vectors and the quantizer
// indices of RPW vectors (D bytes each, one 32-bit word per lane and 4
// positions).  The finished codes are staged in vector 0's buffer, which is
// dead by then (RPW cs <= 4 (D + 12) bytes < its 4 (D + D/8 + 8)).
template <int LOG_D, int RPW>
__host__ __device__ constexpr int encode2_warp_bytes_c() {
    return 4 * RPW * vec_row_floats<(1 << LOG_D)>() + RPW * (1 << LOG_D);
}

template <int LOG_D, bool NIBBLE>
__global__ void __launch_bounds__(32 * enc2_max_warps<LOG_D, NIBBLE>()) encode2_kernel(
    const float *__restrict__ X, size_t n, uint8_t *__restrict__ out, Params P, DevTables T) {
    constexpr int RPW = enc2_rpw<LOG_D, NIBBLE>();  // rows per warp
    constexpr int D = 1 << LOG_D;
    constexpr int E = D / 32;
    constexpr int VS = vec_row_floats<D>();
    static_assert(E >= 8 && E <= 32, "encode2 covers D = 256..1024");
    extern __shared__ __align__(16) unsigned char smem[];
    load_tables(smem, P, T, true, P.qflag != 0);
    float *s_crep = reinterpret_cast<float *>(smem + kTabBytes);  // P.qflag: [levels][32]
    if (P.qflag)
        for (int i = threadIdx.x; i < P.levels * 32; i += blockDim.x) s_crep[i] = T.centroids[i >> 5];
    __syncthreads();
    const float *s_cent = reinterpret_cast<const float *>(smem + kTabCentOff);
    const float *s_bnd = reinterpret_cast<const float *>(smem + kTabBndOff);
    const uint32_t *s_rot = reinterpret_cast<const uint32_t *>(smem + kTabRotOff);
    const uint32_t *s_qjl = reinterpret_cast<const uint32_t *>(smem + kTabQjlOff);
    const uint8_t *s_qlut = smem + kTabQlutOff;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int cs = P.cs;
    unsigned char *wbase = smem + kTabBytes + crep_bytes(P) + warp * encode2_warp_bytes_c<LOG_D, RPW>();
    float *buf = reinterpret_cast<float *>(wbase);
    uint32_t *idxw = reinterpret_cast<uint32_t *>(wbase + 4 * RPW * VS);  // [RPW][E/4][32]
    uint8_t *stage = wbase;  // vector 0's buffer, once phase G has transformed it
    // 8-lane group g runs the reduction chains of row g; with 3 rows per warp
    // group 3 repeats row 2's (its results are not used)
    const int g = lane >> 3;
    const int gv = g < RPW ? g : RPW - 1;
    // sign bits of this lane's layout-A elements lane*E .. lane*E + E-1
    const int bit0 = lane * E;
    const uint32_t emask = (E >= 32) ? 0xffffffffu : ((1u << E) - 1u);
    const uint32_t rbits = (s_rot[bit0 >> 5] >> (bit0 & 31)) & emask;
    const uint32_t qbits = (s_qjl[bit0 >> 5] >> (bit0 & 31)) & emask;
    const bool vec4 = ((P.dim & 3) == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const size_t ngroups = (n + RPW - 1) / RPW;

    // Each warp steps through the phases of its own row groups on its own:
    // the buffers are the warp's and the tables read-only, so the phases are
    // ordered by warp barriers alone, and a warp in a reduction chain overlaps
    // another warp's transforms (block barriers here cost 11%).
    for (size_t base = (size_t)blockIdx.x * nwarps; base < ngroups; base += (size_t)gridDim.x * nwarps) {
        const size_t qd = base + warp;
        const bool active = qd < ngroups;
        const size_t row0 = qd * RPW;
        const int nv = !active ? 0 : ((n - row0 < (size_t)RPW) ? (int)(n - row0) : RPW);
        float norm = 0.0f, inv_norm = 0.0f;
        // the rows of this warp's next group go to L2 while this one is encoded
        if (vec4 && lane == 0) {
            const size_t nrow0 = (qd + (size_t)gridDim.x * nwarps) * RPW;
            if (nrow0 < n) {
                const size_t rows = (n - nrow0 < (size_t)RPW) ? (n - nrow0) : RPW;
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(X + nrow0 * (size_t)P.dim),
                             "r"((uint32_t)(rows * (size_t)P.dim * 4)) : "memory");
            }
        }
        // A: rows -> buffers (zero padded); B: norm
        if (active) {
            if (vec4) {
                // every 16-byte chunk as an async copy (all in flight at
                // once); the zero padding past dim as plain stores
                const int d4 = P.dim >> 2;
#pragma unroll 4
                for (int i = lane; i < RPW * (D / 4); i += 32) {  // i = v * (D/4) + chunk
                    const int v = i / (D / 4), i4 = i % (D / 4);
                    float *dst = buf + v * VS + PadLayout<E>::chunk(i4);
                    if (v < nv && i4 < d4) {
                        const float *src = X + (row0 + v) * (size_t)P.dim + 4 * i4;
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)),
                                     "l"(src) : "memory");
                    } else {
                        *reinterpret_cast<float4 *>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
            } else {
#pragma unroll 1
                for (int v = 0; v < RPW; ++v) {
                    const float *src = X + (row0 + v) * (size_t)P.dim;
#pragma unroll 1
                    for (int i = lane; i < D; i += 32)
                        buf[v * VS + PadLayout<E>::elem(i)] = (v < nv && i < P.dim) ? __ldcs(src + i) : 0.0f;
                }
            }
            __syncwarp();
            const float nsq = chain_sq_reduce2<E, false>(buf + gv * VS, P.dim, lane);
            norm = __fsqrt_rn(nsq);
            inv_norm = (nsq > f32_bits(kNormSqFloorBits)) ? __fdiv_rn(1.0f, norm) : 0.0f;
        }
        __syncwarp();
        // C: rotated = RHT_rot(raw * inv_norm), written back in layout B; D: sigma
        float sigma = 0.0f, inv_sigma = 0.0f;
        if (active) {
#pragma unroll 1
            for (int v = 0; v < RPW; ++v) {
                float *b = buf + v * VS;
                float x[E];
                rht2<E, true>(b, lane, __shfl_sync(kFull, inv_norm, 8 * v), rbits, P.wht_scale, x);
#pragma unroll
                for (int t = 0; t < E; ++t) b[PadLayout<E>::elem(32 * t + lane)] = x[t];
            }
            __syncwarp();
            const float var = chain_sq_reduce2<E, true>(buf + gv * VS, D, lane);
            sigma = __fsqrt_rn(__fdiv_rn(var, (float)D));
            if (f32_bits(kSigmaFloorBits) > sigma) {
                sigma = f32_bits(kSigmaFloorBits);
                inv_sigma = f32_bits(kInvSigmaFloorBits);
            } else {
                inv_sigma = __fdiv_rn(1.0f, sigma);
            }
        }
        __syncwarp();
        // E: quantize + residual in layout B, four indices per lane-word into
        // the per-warp index array; F: gamma
        float gamma = 0.0f;
        if (active) {
            // Every Lloyd-Max table of b = 6..9 has at most one boundary per
            // bucket (qlut_k = 1), and b = 2..5 have at most 15 boundaries:
            // either way no loop over a table (quantize_regs).
            const int qmode = quant_mode(P);
            float breg[15];
            load_bound_regs(breg, P, s_bnd);
#pragma unroll 1
            for (int v = 0; v < RPW; ++v) {
                const float sg = __shfl_sync(kFull, sigma, 8 * v);
                const float isg = __shfl_sync(kFull, inv_sigma, 8 * v);
                float *b = buf + v * VS;
                // This lane's E values are loaded first, quantized in
                // registers and stored afterwards: a store into the buffer
                // between two of its loads would order every element's chain
                // of table loads after the previous one's.
                float xr[E];
                uint32_t wq[E / 4] = {};
#pragma unroll
                for (int t = 0; t < E; ++t) xr[t] = b[PadLayout<E>::elem(32 * t + lane)];
                auto emit = [&](int t, int idx) { wq[t >> 2] |= (uint32_t)idx << (8 * (t & 3)); };
                if (P.qflag)
                    quantize_regs_flag<E>(xr, isg, sg, P, s_bnd, s_qlut, s_crep + lane, emit);
                else
                    quantize_regs<E>(xr, isg, sg, qmode, P, breg, s_bnd, s_qlut, s_cent, emit);
#pragma unroll
                for (int t = 0; t < E; ++t) b[PadLayout<E>::elem(32 * t + lane)] = xr[t];
#pragma unroll
                for (int t4 = 0; t4 < E / 4; ++t4) idxw[(v * (E / 4) + t4) * 32 + lane] = wq[t4];
            }
            __syncwarp();
            gamma = __fsqrt_rn(chain_sq_reduce2<E, true>(buf + gv * VS, D, lane));
        }
        __syncwarp();
        // G: RHT_qjl(residual), pack units + trailer; H: staged codes -> global
        if (active) {
#pragma unroll 1
            for (int v = 0; v < nv; ++v) {
                float x[E];
                rht2<E, false>(buf + v * VS, lane, 1.0f, qbits, P.wht_scale, x);
                uint8_t *st = stage + v * cs;
                uint32_t wq[E / 4];  // all index words first: no load after a store
#pragma unroll
                for (int t4 = 0; t4 < E / 4; ++t4) wq[t4] = idxw[(v * (E / 4) + t4) * 32 + lane];
#pragma unroll
                for (int t4 = 0; t4 < E / 4; ++t4) {
                    const uint32_t word = wq[t4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int t = 4 * t4 + q;
                        const uint32_t idx = (word >> (8 * q)) & 0xFFu;
                        const uint32_t unit = ((idx << 1) | (x[t] >= 0.0f ? 1u : 0u)) & 0xFFu;
                        const int e = 32 * t + lane;
                        if constexpr (NIBBLE) {
                            const uint32_t up = __shfl_down_sync(kFull, unit, 1);
                            if (!(lane & 1)) st[e >> 1] = (uint8_t)((unit | (up << 4)) & 0xFFu);
                        } else {
                            st[e] = (uint8_t)unit;
                        }
                    }
                }
            }
            if ((lane & 7) == 0 && g < nv) {
                uint8_t *t = stage + g * cs + P.pb;
                const uint32_t w[3] = {__float_as_uint(norm), __float_as_uint(gamma), __float_as_uint(sigma)};
#pragma unroll
                for (int q = 0; q < 12; ++q) t[q] = (uint8_t)(w[q >> 2] >> (8 * (q & 3)));
            }
            __syncwarp();
            uint8_t *dst = out + row0 * (size_t)cs;
            const int len = nv * cs;
            if (((reinterpret_cast<uintptr_t>(dst) & 15) == 0) && ((len & 15) == 0)) {
                const uint4 *s4 = reinterpret_cast<const uint4 *>(stage);
                uint4 *d4 = reinterpret_cast<uint4 *>(dst);
#pragma unroll 1
                for (int i = lane; i < (len >> 4); i += 32) __stcs(d4 + i, s4[i]);
            } else if (((reinterpret_cast<uintptr_t>(dst) & 3) == 0) && ((len & 3) == 0)) {
                // groups of 3 codes of 4k + 12 bytes start on 4-byte boundaries
                const uint32_t *s1 = reinterpret_cast<const uint32_t *>(stage);
                uint32_t *d1 = reinterpret_cast<uint32_t *>(dst);
#pragma unroll 1
                for (int i = lane; i < (len >> 2); i += 32) __stcs(d1 + i, s1[i]);
            } else {
#pragma unroll 1
                for (int i = lane; i < len; i += 32) dst[i] = stage[i];
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// prepareQuery: one warp per query.
// ---------------------------------------------------------------------------
template <int LOG_D>
__global__ void __launch_bounds__(256) prepare_kernel(const float *__restrict__ Q, size_t m,
                                                      float *__restrict__ q_rot,
                                                      float *__restrict__ s_q,
                                                      float *__restrict__ norms, Params P,
                                                      DevTables T) {
    constexpr int D = 1 << LOG_D;
    constexpr int VS = D + 8;
    extern __shared__ __align__(16) unsigned char smem[];
    load_tables(smem, P, T, false);
    __syncthreads();
    const uint32_t *s_rot = reinterpret_cast<const uint32_t *>(smem + kTabRotOff);
    const uint32_t *s_qjl = reinterpret_cast<const uint32_t *>(smem + kTabQjlOff);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    float *buf = reinterpret_cast<float *>(smem + kTabBytes) + warp * VS;
    for (size_t qi = (size_t)blockIdx.x * nwarps + warp; qi < m; qi += (size_t)gridDim.x * nwarps) {
        const float *src = Q + qi * (size_t)P.dim;
        for (int i = lane; i < D; i += 32) buf[swz(i)] = (i < P.dim) ? src[i] : 0.0f;
        __syncwarp();
        // |q|^2: the reference's batch drivers evaluate this loop as a plain
        // sequential sum (:443-445).  Lane 0 keeps the order; the squares of
        // each run of 32 elements are formed by their lanes and handed over
        // by shuffles, so the chain waits only on its adds.
        float qn2 = 0.0f;
        for (int i0 = 0; i0 < P.dim; i0 += 32) {
            const int i = i0 + lane;
            const float x = (i < P.dim) ? buf[swz(i)] : 0.0f;
            const float sq = __fmul_rn(x, x);
            const int cnt = (P.dim - i0 < 32) ? (P.dim - i0) : 32;
#pragma unroll
            for (int t = 0; t < 32; ++t) {
                const float v = __shfl_sync(kFull, sq, t);
                if (t < cnt) qn2 = __fadd_rn(qn2, v);
            }
        }
        const float qn = __fsqrt_rn(qn2);
        const float qinv = (qn2 > f32_bits(kNormSqFloorBits)) ? __fdiv_rn(1.0f, qn) : 0.0f;
        fwht_from<LOG_D, 0, true>(buf, lane, qinv, s_rot, P.wht_scale);
        float *qr = q_rot + qi * (size_t)D;
        for (int i = lane; i < D; i += 32) qr[i] = buf[swz(i)];
        fwht_from<LOG_D, 0, false>(buf, lane, 1.0f, s_qjl, P.wht_scale);
        float *sq = s_q + qi * (size_t)D;
        for (int i = lane; i < D; i += 32) sq[i] = buf[swz(i)];
        if (lane == 0) {
            norms[2 * qi] = qn2;
            norms[2 * qi + 1] = qn;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// scan: row i of the query side (blockIdx.y) against a stream of n codes.
//   SYM = false: asymmetric distSearch; the row is a prepared query
//                (q_rot, s_q, |q|^2, |q|).
//   SYM = true:  MSE-only distBuild; the row is code a_i, decoded to
//                c[idx] * sigma_a per coordinate.
// A code of PB packed bytes is read as W = PB/4 32-bit words by LPC lanes
// (WPL words each, coalesced); CPS codes share a warp step.  The query side
// of each lane's positions sits in registers; centroids come from a
// lane-replicated shared table (entry v of lane l at v*32 + l: conflict-free).
// ---------------------------------------------------------------------------
template <int LOG_D, bool NIBBLE>
struct ScanShape {
    static constexpr int D = 1 << LOG_D;
    static constexpr int PB = NIBBLE ? D / 2 : D;
    static constexpr int W = PB / 4;
    static constexpr int LPC = W < 1 ? 1 : (W < 32 ? W : 32);
    static constexpr int WPL = W / LPC;
    static constexpr int CPS = 32 / LPC;
    static constexpr int PPW = NIBBLE ? 8 : 4;
    static constexpr int PPL = WPL * PPW;
    static constexpr bool QREG = PPL <= 32;
    static constexpr int U = QREG ? (WPL >= 8 ? 2 : 4) : 1;  // warp steps per iteration
};

template <int LOG_D, bool NIBBLE>
__device__ __forceinline__ unsigned unit_of(uint32_t w, int b) {
    return NIBBLE ? ((w >> (4 * b)) & 15u) : ((w >> (8 * b)) & 255u);
}

template <int LOG_D, bool NIBBLE, bool SYM>
__global__ void __launch_bounds__(256) scan_kernel(const float *__restrict__ q_rot,
                                                   const float *__restrict__ s_q,
                                                   const float *__restrict__ norms,
                                                   const uint8_t *__restrict__ codes_a,
                                                   const uint8_t *__restrict__ codes, size_t n,
                                                   float *__restrict__ out, size_t ldo, Params P,
                                                   DevTables T) {
    using S = ScanShape<LOG_D, NIBBLE>;
    constexpr int PPL = S::PPL;
    constexpr int NQ = S::QREG ? PPL : 1;
    extern __shared__ __align__(16) float fsm[];
    // one entry per value of (unit >> 1) a code byte can hold: 8 (nibble) or
    // 128 (byte); entries past the table's levels read as 0
    constexpr int LUTN = NIBBLE ? 8 : 128;
    float *s_lut = fsm;                          // [LUTN * 32]
    float *s_qa = fsm + LUTN * 32;               // !QREG: [PPL * 32] query side (q_rot or a)
    float *s_qb = s_qa + (S::QREG ? 0 : PPL * 32);  // !QREG: [PPL * 32] -s_q
    const int tid = threadIdx.x, lane = tid & 31;
    const int sl = lane % S::LPC, slot = lane / S::LPC;
    const size_t row = blockIdx.y;
    const int cs = P.cs;
    for (int i = tid; i < LUTN * 32; i += blockDim.x) s_lut[i] = T.centroids[i >> 5];

    // query side of this lane's positions p(j, b) = PPW * (sl + LPC * j) + b
    float qa[NQ], qb[NQ];
    float rn2 = 0.0f, rn = 0.0f;
    if constexpr (!SYM) {
        const float *qr = q_rot + row * (size_t)S::D;
        const float *sq = s_q + row * (size_t)S::D;
        rn2 = norms[2 * row];
        rn = norms[2 * row + 1];
#pragma unroll
        for (int j = 0; j < S::WPL; ++j)
#pragma unroll
            for (int b = 0; b < S::PPW; ++b) {
                const int p = S::PPW * (sl + S::LPC * j) + b;
                const int r = j * S::PPW + b;
                if constexpr (S::QREG) {
                    qa[r] = qr[p];
                    qb[r] = -sq[p];
                } else if (tid < 32) {
                    s_qa[r * 32 + lane] = qr[p];
                    s_qb[r * 32 + lane] = -sq[p];
                }
            }
    } else {
        const uint8_t *ca = codes_a + row * (size_t)cs;
        const float *ma = reinterpret_cast<const float *>(ca + S::PB);
        const float sig_a = ma[2];
        rn = ma[0];
        rn2 = __fmul_rn(rn, rn);
#pragma unroll
        for (int j = 0; j < S::WPL; ++j) {
            const uint32_t w = reinterpret_cast<const uint32_t *>(ca)[sl + S::LPC * j];
#pragma unroll
            for (int b = 0; b < S::PPW; ++b) {
                const int r = j * S::PPW + b;
                const float v = __fmul_rn(T.centroids[unit_of<LOG_D, NIBBLE>(w, b) >> 1], sig_a);
                if constexpr (S::QREG) qa[r] = v;
                else if (tid < 32) s_qa[r * 32 + lane] = v;
            }
        }
    }
    __syncthreads();

    const size_t warps_total = (size_t)gridDim.x * (blockDim.x >> 5);
    const size_t wg = (size_t)blockIdx.x * (blockDim.x >> 5) + (tid >> 5);
    float *orow = out + row * ldo;
    constexpr int STEP = S::CPS * S::U;
    for (size_t c0 = wg * STEP; c0 < n; c0 += warps_total * STEP) {
        uint32_t w[S::U][S::WPL];
        float sig_b[S::U];
#pragma unroll
        for (int u = 0; u < S::U; ++u) {
            const size_t c = c0 + (size_t)u * S::CPS + slot;
            const uint32_t *cw = reinterpret_cast<const uint32_t *>(codes + c * (size_t)cs);
#pragma unroll
            for (int j = 0; j < S::WPL; ++j) w[u][j] = (c < n) ? __ldg(cw + sl + S::LPC * j) : 0u;
            if constexpr (SYM)
                sig_b[u] = (c < n) ? __ldg(reinterpret_cast<const float *>(cw + S::W) + 2) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < S::U; ++u) {
            float ip = 0.0f, dot = 0.0f;
#pragma unroll
            for (int j = 0; j < S::WPL; ++j) {
#pragma unroll
                for (int b = 0; b < S::PPW; ++b) {
                    const int r = j * S::PPW + b;
                    const unsigned un = unit_of<LOG_D, NIBBLE>(w[u][j], b);
                    const float cv = s_lut[((un >> 1) << 5) + lane];
                    const float a = S::QREG ? qa[r] : s_qa[r * 32 + lane];
                    if constexpr (SYM) {
                        // (c[a] sigma_a) * (c[b] sigma_b), each factor rounded (:709-710)
                        ip = __fmaf_rn(a, __fmul_rn(cv, sig_b[u]), ip);
                    } else {
                        ip = __fmaf_rn(a, cv, ip);
                        const float nb = S::QREG ? qb[r] : s_qb[r * 32 + lane];
                        dot = __fadd_rn(dot, __uint_as_float(__float_as_uint(nb) ^ ((un & 1u) << 31)));
                    }
                }
            }
#pragma unroll
            for (int off = S::LPC / 2; off > 0; off >>= 1) {
                ip = __fadd_rn(ip, __shfl_xor_sync(kFull, ip, off));
                if constexpr (!SYM) dot = __fadd_rn(dot, __shfl_xor_sync(kFull, dot, off));
            }
            const size_t c = c0 + (size_t)u * S::CPS + slot;
            if (sl == 0 && c < n) {
                const float *meta = reinterpret_cast<const float *>(codes + c * (size_t)cs + S::PB);
                const float xn = meta[0];
                float d;
                if constexpr (SYM) {
                    const float ipt = __fmul_rn(__fmul_rn(ip, rn), xn);  // ip_rot * n_a * n_b
                    d = __fsub_rn(__fadd_rn(rn2, __fmul_rn(xn, xn)), __fmul_rn(2.0f, ipt));
                } else {
                    const float ip_mse = __fmul_rn(ip, meta[2]);
                    const float corr = __fmul_rn(__fmul_rn(P.scale, meta[1]), dot);
                    const float ipt = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), xn), rn);
                    d = __fsub_rn(__fadd_rn(rn2, __fmul_rn(xn, xn)), __fmul_rn(2.0f, ipt));
                }
                orow[c] = d > 0.0f ? d : 0.0f;
            }
        }
    }
}

// Packed FP32x2 FMA (two independent IEEE FMAs on a register pair).
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float sum2(unsigned long long v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return lo + hi;
}

// ---------------------------------------------------------------------------
// The byte-unit scan arithmetic (bits >= 5, D = 128 * WPL), shared by scan8b
// and the staged scan (scan8_setup / scan8_terms).
// A code is read as D/4 32-bit words, word l + 32 j by lane l; each lane owns
// positions p = 4 (l + 32 j) + b and keeps q_rot[p] in registers.
//   centroid term: shared memory holds one 256-byte row per unit byte u whose
//     first 128 bytes are c[u >> 1] replicated in 32 lane columns, so each
//     position costs one PRMT (byte -> row | lane column) and one
//     bank-conflict-free LDS, then an FFMA;
//   QJL term: s_q is held per query as 16-bit fixed point, s_q ~ step * s16,
//     split into a signed high byte and an unsigned low byte packed four per
//     register; the four sign bits of a word are its bytes & 1, so
//     sum_p bit_p s16_p costs two dp4a per word and
//     dot = step * (2 sum_p bit_p s16_p - sum_p s16_p).
//     The fixed-point error enters only the correction term scale*gamma*dot
//     (space_turbo_quant.h:683), where it is below 1e-6 of the distance's
//     term scale at the sizes used here.
template <int WPL>
struct Scan8Query {
    unsigned long long qr2[2 * WPL];  // q_rot of positions 4 (lane + 32 j) + {0,1}, {2,3}
    int shi[WPL];                     // s_q fixed point, signed high bytes
    unsigned slo[WPL];                // s_q fixed point, unsigned low bytes
};

// Per-query set-up shared by the byte-unit scans: the lane-replicated centroid
// table (256 rows of 256 bytes, entry of lane l at row * 256 + 4 l), the
// fixed-point step of s_q (max |s_q| / 32767), this lane's query registers and
// the sum of all fixed-point s_q.  Ends with a block barrier.
template <int WPL>
__device__ __forceinline__ void scan8_setup(const float *__restrict__ qr_g,
                                            const float *__restrict__ sq_g, unsigned char *tab,
                                            const DevTables &T, float *s_red, Scan8Query<WPL> &Q,
                                            int &ssum, float &step) {
    constexpr int D = 128 * WPL;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int i = tid; i < 256 * 32; i += blockDim.x)
        reinterpret_cast<float *>(tab + (i >> 5) * 256)[i & 31] = T.centroids[(i >> 5) >> 1];
    float mx = 0.0f;
    for (int i = tid; i < D; i += blockDim.x) mx = fmaxf(mx, fabsf(sq_g[i]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, off));
    if (lane == 0) s_red[warp] = mx;
    __syncthreads();
    mx = s_red[0];
    for (int k = 1; k < nw; ++k) mx = fmaxf(mx, s_red[k]);
    step = (mx > 0.0f) ? mx / 32767.0f : 1.0f;
    const float inv_step = 1.0f / step;
    int sum = 0;
#pragma unroll
    for (int j = 0; j < WPL; ++j) {
        unsigned hi = 0, lo = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int p = 4 * (lane + 32 * j) + b;
            if (b & 1) Q.qr2[2 * j + (b >> 1)] = pack2(qr_g[p - 1], qr_g[p]);
            int v = __float2int_rn(sq_g[p] * inv_step);
            v = max(-32767, min(32767, v));
            sum += v;
            hi |= ((unsigned)(v >> 8) & 0xFFu) << (8 * b);
            lo |= ((unsigned)v & 0xFFu) << (8 * b);
        }
        Q.shi[j] = (int)hi;
        Q.slo[j] = lo;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
    ssum = sum;
    __syncthreads();
}

// This lane's share of one code: the centroid dot over its 4 WPL positions and
// the fixed-point sign sum (exact integer, |.| < 2^21).
template <int WPL, bool PACK>
__device__ __forceinline__ void scan8_terms(const uint32_t (&w)[WPL], const Scan8Query<WPL> &Q,
                                            const unsigned char *tab, uint32_t lane4, float &ip,
                                            float &sg) {
    int acc_hi = 0;
    unsigned acc_lo = 0;
    if constexpr (PACK) {
        unsigned long long acc2 = 0ull;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
            const uint32_t x = w[j];
            float cv[4];
#pragma unroll
            for (int b = 0; b < 4; ++b)
                cv[b] = *reinterpret_cast<const float *>(
                    tab + __byte_perm(x, lane4, 0x6504u | ((uint32_t)b << 4)));
            acc2 = ffma2(Q.qr2[2 * j], pack2(cv[0], cv[1]), acc2);
            acc2 = ffma2(Q.qr2[2 * j + 1], pack2(cv[2], cv[3]), acc2);
            const uint32_t bits = x & 0x01010101u;
            acc_hi = __dp4a((int)bits, Q.shi[j], acc_hi);
            acc_lo = __dp4a(bits, Q.slo[j], acc_lo);
        }
        ip = sum2(acc2);
    } else {
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
            const uint32_t x = w[j];
            float q[4];
            asm("mov.b64 {%0, %1}, %2;" : "=f"(q[0]), "=f"(q[1]) : "l"(Q.qr2[2 * j]));
            asm("mov.b64 {%0, %1}, %2;" : "=f"(q[2]), "=f"(q[3]) : "l"(Q.qr2[2 * j + 1]));
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const float c = *reinterpret_cast<const float *>(
                    tab + __byte_perm(x, lane4, 0x6504u | ((uint32_t)b << 4)));
                if (b & 1) a1 = __fmaf_rn(q[b], c, a1);
                else a0 = __fmaf_rn(q[b], c, a0);
            }
            const uint32_t bits = x & 0x01010101u;
            acc_hi = __dp4a((int)bits, Q.shi[j], acc_hi);
            acc_lo = __dp4a(bits, Q.slo[j], acc_lo);
        }
        ip = a0 + a1;
    }
    sg = (float)(acc_hi * 256 + (int)acc_lo);
}

// Transpose reduction of 8 values over the warp (9 shuffles).  On return every
// lane holds the warp sum of value 4 b4 + 2 b3 + b2 (b_i = bit i of the lane).
__device__ __forceinline__ float transpose8(const float (&v)[8], int lane) {
    float a[4];
    const bool h16 = lane & 16;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float send = h16 ? v[k] : v[k + 4];
        const float keep = h16 ? v[k + 4] : v[k];
        a[k] = keep + __shfl_xor_sync(kFull, send, 16);
    }
    float b[2];
    const bool h8 = lane & 8;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float send = h8 ? a[k] : a[k + 2];
        const float keep = h8 ? a[k + 2] : a[k];
        b[k] = keep + __shfl_xor_sync(kFull, send, 8);
    }
    const bool h4 = lane & 4;
    float y = (h4 ? b[1] : b[0]) + __shfl_xor_sync(kFull, h4 ? b[0] : b[1], 4);
    y += __shfl_xor_sync(kFull, y, 2);
    y += __shfl_xor_sync(kFull, y, 1);
    return y;
}

// The reference's distance epilogue (distSearch*, space_turbo_quant.h:683-685)
// from the reduced centroid dot `ipr`, the fixed-point sign sum `sb` and the
// code's trailer (norm t0, gamma t1, sigma t2).
__device__ __forceinline__ float scan8_distance(float ipr, float sb, float t0, float t1, float t2,
                                                float step, int ssum, float sc, float qn2,
                                                float qn) {
    const float dot = __fmul_rn(step, 2.0f * sb - (float)ssum);
    const float ip_mse = __fmul_rn(ipr, t2);
    const float corr = __fmul_rn(__fmul_rn(sc, t1), dot);
    const float ipt = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), t0), qn);
    const float d = __fsub_rn(__fadd_rn(qn2, __fmul_rn(t0, t0)), __fmul_rn(2.0f, ipt));
    return d > 0.0f ? d : 0.0f;
}

// ---------------------------------------------------------------------------
// scan8b: that arithmetic with registers fed by plain loads (any 4-byte
// aligned corpus; query rows on grid.y).  A warp owns batches of 16
// consecutive codes and runs them as 8 steps of 2 codes; the word registers of
// the next step are loaded (ping-pong, no copies) before the current step is
// reduced, and code indices past the end are clamped to the last code, so the
// loads need no bounds checks.  After each step's transpose reduction the
// 8-lane group holding a value keeps it in the lane whose (lane & 7) is the
// step, so after 8 steps lane l holds value kind (l >> 3) & 1 of code
// 2 (l & 7) + (l >> 4): 16 lanes then finish the 16 codes together (trailer
// loaded at the start of the batch, one store each).  Per code this is the
// same sequence of roundings as the staged scan's byte units.
// ---------------------------------------------------------------------------
template <int WPL>
__global__ void __launch_bounds__(256, 2) scan8b_kernel(const float *__restrict__ q_rot,
                                                        const float *__restrict__ s_q,
                                                        const float *__restrict__ norms,
                                                        const uint8_t *__restrict__ codes, size_t n,
                                                        float *__restrict__ out, size_t ldo, Params P,
                                                        DevTables T) {
    constexpr int D = 128 * WPL;
    extern __shared__ __align__(16) unsigned char tab[];
    __shared__ float s_red[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const size_t row = blockIdx.y;
    Scan8Query<WPL> Q;
    int ssum;
    float step;
    scan8_setup<WPL>(q_rot + row * (size_t)D, s_q + row * (size_t)D, tab, T, s_red, Q, ssum, step);
    const float qn2 = norms[2 * row], qn = norms[2 * row + 1];
    const float sc = P.scale;

    const uint32_t lane4 = (uint32_t)lane * 4u;
    const size_t cs = (size_t)P.cs;
    const size_t last = n - 1;
    const size_t nbatch = (n + 15) >> 4;
    const size_t bstride = (size_t)gridDim.x * nw;
    size_t bt = (size_t)blockIdx.x * nw + warp;
    if (bt >= nbatch) return;
    const int ecode = 2 * (lane & 7) + (lane >> 4);  // the code this lane finishes
    const bool eowner = !(lane & 8);
    float *orow = out + row * ldo;

    auto load = [&](uint32_t (&w)[2][WPL], size_t c0) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const size_t c = (c0 + u < last) ? c0 + u : last;
            const uint32_t *cw = reinterpret_cast<const uint32_t *>(codes + c * cs);
#pragma unroll
            for (int j = 0; j < WPL; ++j) w[u][j] = __ldg(cw + lane + 32 * j);
        }
    };
    // one step: 2 codes -> the transpose-reduced value of this lane's group
    auto reduce_step = [&](const uint32_t (&w)[2][WPL]) -> float {
        float v[4];
#pragma unroll
        for (int u = 0; u < 2; ++u) scan8_terms<WPL, true>(w[u], Q, tab, lane4, v[2 * u], v[2 * u + 1]);
        float w2[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const bool hi = lane & 16;
            const float send = hi ? v[k] : v[k + 2];
            const float keep = hi ? v[k + 2] : v[k];
            w2[k] = keep + __shfl_xor_sync(kFull, send, 16);
        }
        float y;
        {
            const bool hi = lane & 8;
            const float send = hi ? w2[0] : w2[1];
            const float keep = hi ? w2[1] : w2[0];
            y = keep + __shfl_xor_sync(kFull, send, 8);
        }
        y += __shfl_xor_sync(kFull, y, 4);
        y += __shfl_xor_sync(kFull, y, 2);
        y += __shfl_xor_sync(kFull, y, 1);
        return y;
    };

    uint32_t wa[2][WPL], wb[2][WPL];
    load(wa, bt << 4);
    for (;;) {
        const size_t cbase = bt << 4;
        const size_t next_bt = bt + bstride;
        // trailer of the code this lane finishes (used after the 8 steps)
        const size_t ce = cbase + (size_t)ecode;
        const float *tm = reinterpret_cast<const float *>(codes + (ce < last ? ce : last) * cs + D);
        const float t0 = __ldg(tm), t1 = __ldg(tm + 1), t2 = __ldg(tm + 2);
        float R = 0.0f;
#pragma unroll 1
        for (int s = 0; s < 8; s += 2) {
            load(wb, cbase + 2 * s + 2);
            const float ya = reduce_step(wa);
            R = ((lane & 7) == s) ? ya : R;
            load(wa, (s + 2 < 8) ? cbase + 2 * s + 4 : (next_bt << 4));
            const float yb = reduce_step(wb);
            R = ((lane & 7) == s + 1) ? yb : R;
        }
        const float sb = __shfl_down_sync(kFull, R, 8);
        if (eowner && ce < n) orow[ce] = scan8_distance(R, sb, t0, t1, t2, step, ssum, sc, qn2, qn);
        bt = next_bt;
        if (bt >= nbatch) break;
    }
}

// ---------------------------------------------------------------------------
// scan8t: the 1->N byte-unit scan (scan8's arithmetic) fed from shared memory.
// The corpus is read as groups of 4 consecutive codes: 4 cs bytes, a multiple
// of 16, so a group is one untiled bulk copy.  Warp w of the grid owns groups
// w, w + TW, w + 2 TW, ... (TW = warps in the grid) and streams them with
// cp.async.bulk into a private ring of S stages, one mbarrier per stage; lane
// 0 refills a stage as soon as the warp has read it.  The bytes in flight per
// SM are therefore set by the rings (NW x (S - 1) groups), not by registers.
// Lane l reads word l + 32 j of every code from shared memory: consecutive
// words, so the reads are conflict-free at any code offset.
// Each stage gives 8 values (centroid dot and sign sum of 4 codes) that one
// transpose reduction leaves in the lane groups of 4; across a batch of 4
// stages lane l keeps the value of stage l & 3, and the 16 lanes with bit 2
// clear then finish the batch's 16 codes (trailer, distance, store).
// The last n mod 4 codes are read with plain loads by the warp that would own
// group n / 4.  The caller guarantees a 16-byte aligned corpus.
// ---------------------------------------------------------------------------
constexpr int kErrScanWait = 5;  // status code: a scan stage never arrived

// ---------------------------------------------------------------------------
// Unit policies of the staged scan.  A code's packed part is PB = 128 WPL
// bytes, read by lane l as words l + 32 j (j < WPL).
//   ByteUnits   (bits >= 5, D = 128 WPL): one unit per byte; one 4-byte lookup
//               per coordinate (scan8_terms).
//   NibbleUnits (bits <= 4, D = 256 WPL): two units per byte; the table row of
//               byte value u holds the pair (c[lo >> 1], c[hi >> 1]) of its
//               low and high nibble in each lane column (8 bytes), so one
//               8-byte lookup gives both coordinates of a byte and feeds a
//               packed FP32x2 FMA with the query pair (q[2b], q[2b + 1]).
// Both tables are 256 rows x 256 bytes (64 KB), lane-replicated.
// ---------------------------------------------------------------------------
// A group of 4 codes with a whole warp per code (lane l reads words
// l + 32 j): 8 values (centroid dot, sign sum of each code) reduced by one
// transpose; value 2 c + kind of code c ends in the lanes with
// 2 b4 + b3 = c, b2 = kind.  word(c, i) returns word i of code c.
template <class U, class Word>
__device__ __forceinline__ float full_warp_group(Word word, const typename U::Query &Q,
                                                 const unsigned char *tab, int lane) {
    constexpr int WPL = U::kWPL;
    uint32_t w[4][WPL];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int j = 0; j < WPL; ++j) w[c][j] = word(c, lane + 32 * j);
    float v[8];
#pragma unroll
    for (int c = 0; c < 4; ++c) U::terms(w[c], Q, tab, lane, v[2 * c], v[2 * c + 1]);
    return transpose8(v, lane);
}

template <int WPL>
struct ByteUnits {
    static constexpr int kWPL = WPL, PB = 128 * WPL;
    using Query = Scan8Query<WPL>;
    __device__ static __forceinline__ void setup(const float *qr, const float *sq, unsigned char *tab,
                                                 const DevTables &T, float *s_red, Query &Q,
                                                 int &ssum, float &step) {
        scan8_setup<WPL>(qr, sq, tab, T, s_red, Q, ssum, step);
    }
    // Scalar FMAs into an even and an odd accumulator: the same operations in the
    // same order as the packed FP32x2 form (each half of fma.rn.f32x2 is one
    // IEEE FMA), so the distances are identical; in this kernel the scalar form
    // takes about 2% fewer cycles per launch and spills nothing.
    __device__ static __forceinline__ void terms(const uint32_t (&w)[WPL], const Query &Q,
                                                 const unsigned char *tab, int lane, float &ip,
                                                 float &sg) {
        scan8_terms<WPL, false>(w, Q, tab, (uint32_t)lane * 4u, ip, sg);
    }
    template <class Word>
    __device__ static __forceinline__ float group(Word word, const Query &Q,
                                                  const unsigned char *tab, int lane) {
        return full_warp_group<ByteUnits<WPL>>(word, Q, tab, lane);
    }
    __device__ static __forceinline__ int code_of_lane(int lane) {
        return 2 * ((lane >> 4) & 1) + ((lane >> 3) & 1);
    }
};

template <int WPL>
struct NibbleQuery {
    unsigned long long qr2[4 * WPL];  // (q[2b], q[2b + 1]) of byte b = 4 (lane + 32 j) + k
    int she[WPL], sho[WPL];           // s_q fixed point of the even / odd coordinates, high bytes
    unsigned sle[WPL], slo[WPL];      // ... low bytes
};

template <int WPL>
struct NibbleUnits {
    static constexpr int kWPL = WPL, PB = 128 * WPL;
    static constexpr int D = 256 * WPL;
    using Query = NibbleQuery<WPL>;
    __device__ static __forceinline__ void setup(const float *qr_g, const float *sq_g,
                                                 unsigned char *tab, const DevTables &T,
                                                 float *s_red, Query &Q, int &ssum, float &step) {
        setup_lanes(qr_g, sq_g, tab, T, s_red, Q, ssum, step, D, 31);
    }
    // dn: padded dim; lmask: the lane's word column is lane & lmask (31, or 15
    // when half-warps share positions; then lanes >= 16 add nothing to ssum)
    __device__ static __forceinline__ void setup_lanes(const float *qr_g, const float *sq_g,
                                                       unsigned char *tab, const DevTables &T,
                                                       float *s_red, Query &Q, int &ssum,
                                                       float &step, int dn, int lmask) {
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
        const int col = lane & lmask;
        for (int i = tid; i < 256 * 64; i += blockDim.x) {
            const int u = i >> 6, half = i & 1;  // row u, float (lane, half) of the row
            const int unit = half ? (u >> 4) : (u & 15);
            reinterpret_cast<float *>(tab + u * 256)[i & 63] = T.centroids[unit >> 1];
        }
        float mx = 0.0f;
        for (int i = tid; i < dn; i += blockDim.x) mx = fmaxf(mx, fabsf(sq_g[i]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, off));
        if (lane == 0) s_red[warp] = mx;
        __syncthreads();
        mx = s_red[0];
        for (int k = 1; k < nw; ++k) mx = fmaxf(mx, s_red[k]);
        step = (mx > 0.0f) ? mx / 32767.0f : 1.0f;
        const float inv_step = 1.0f / step;
        int sum = 0;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
            unsigned eh = 0, el = 0, oh = 0, ol = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int b = 4 * (col + 32 * j) + k;
                Q.qr2[4 * j + k] = pack2(qr_g[2 * b], qr_g[2 * b + 1]);
                int ve = __float2int_rn(sq_g[2 * b] * inv_step);
                int vo = __float2int_rn(sq_g[2 * b + 1] * inv_step);
                ve = max(-32767, min(32767, ve));
                vo = max(-32767, min(32767, vo));
                sum += ve + vo;
                eh |= ((unsigned)(ve >> 8) & 0xFFu) << (8 * k);
                el |= ((unsigned)ve & 0xFFu) << (8 * k);
                oh |= ((unsigned)(vo >> 8) & 0xFFu) << (8 * k);
                ol |= ((unsigned)vo & 0xFFu) << (8 * k);
            }
            Q.she[j] = (int)eh;
            Q.sle[j] = el;
            Q.sho[j] = (int)oh;
            Q.slo[j] = ol;
        }
        if (lane != col) sum = 0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(kFull, sum, off);
        ssum = sum;
        __syncthreads();
    }
    __device__ static __forceinline__ void terms(const uint32_t (&w)[WPL], const Query &Q,
                                                 const unsigned char *tab, int lane, float &ip,
                                                 float &sg) {
        const uint32_t lane8 = (uint32_t)lane * 8u;
        unsigned long long acc2 = 0ull;
        int acc_hi = 0;
        unsigned acc_lo = 0;
#pragma unroll
        for (int j = 0; j < WPL; ++j) {
            const uint32_t x = w[j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const unsigned long long cv = *reinterpret_cast<const unsigned long long *>(
                    tab + __byte_perm(x, lane8, 0x6504u | ((uint32_t)k << 4)));
                acc2 = ffma2(Q.qr2[4 * j + k], cv, acc2);
            }
            const uint32_t be = x & 0x01010101u, bo = (x >> 4) & 0x01010101u;
            acc_hi = __dp4a((int)be, Q.she[j], acc_hi);
            acc_lo = __dp4a(be, Q.sle[j], acc_lo);
            acc_hi = __dp4a((int)bo, Q.sho[j], acc_hi);
            acc_lo = __dp4a(bo, Q.slo[j], acc_lo);
        }
        ip = sum2(acc2);
        sg = (float)(acc_hi * 256 + (int)acc_lo);  // exact: |.| < 2^22
    }
    template <class Word>
    __device__ static __forceinline__ float group(Word word, const Query &Q,
                                                  const unsigned char *tab, int lane) {
        return full_warp_group<NibbleUnits<WPL>>(word, Q, tab, lane);
    }
    __device__ static __forceinline__ int code_of_lane(int lane) {
        return 2 * ((lane >> 4) & 1) + ((lane >> 3) & 1);
    }
};

// Nibble units at D = 128: a code is 64 packed bytes, 16 words, so a
// half-warp takes one code: lane l reads word l & 15 of code 2 r + (l >> 4) of
// the group (rows r = 0, 1).  The 4 values of a lane (dot and sign sum of its
// two codes) are reduced within the half-warps; value (row b3, kind b2) of
// code 2 b3 + b4 ends in the lane groups of 4 as in full_warp_group.
struct HalfNibbleUnits {
    static constexpr int kWPL = 1, PB = 64, D = 128;
    using Query = NibbleQuery<1>;
    __device__ static __forceinline__ void setup(const float *qr_g, const float *sq_g,
                                                 unsigned char *tab, const DevTables &T,
                                                 float *s_red, Query &Q, int &ssum, float &step) {
        // the half-warps hold the same positions: lane & 15 in NibbleUnits<1>'s
        // layout, and the sign sum counts each position once
        NibbleUnits<1>::setup_lanes(qr_g, sq_g, tab, T, s_red, Q, ssum, step, 128, 15);
    }
    template <class Word>
    __device__ static __forceinline__ float group(Word word, const Query &Q,
                                                  const unsigned char *tab, int lane) {
        float v[4];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t w[1] = {word(2 * r + (lane >> 4), lane & 15)};
            NibbleUnits<1>::terms(w, Q, tab, lane, v[2 * r], v[2 * r + 1]);
        }
        float a[2];
        const bool h8 = lane & 8;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const float send = h8 ? v[k] : v[k + 2];
            const float keep = h8 ? v[k + 2] : v[k];
            a[k] = keep + __shfl_xor_sync(kFull, send, 8);
        }
        const bool h4 = lane & 4;
        float y = (h4 ? a[1] : a[0]) + __shfl_xor_sync(kFull, h4 ? a[0] : a[1], 4);
        y += __shfl_xor_sync(kFull, y, 2);
        y += __shfl_xor_sync(kFull, y, 1);
        return y;
    }
    __device__ static __forceinline__ int code_of_lane(int lane) {
        return 2 * ((lane >> 3) & 1) + ((lane >> 4) & 1);
    }
};

// Groups of 4 codes per ring stage: small codes are fetched several groups
// at a time so that each bulk copy moves ~2 KB or more.
template <int PB>
constexpr int scant_gps() {
    return (4 * (PB + 12) >= 2048) ? 1 : ((4 * (PB + 12) >= 1024) ? 2 : 4);
}

// Stages of a warp ring of about `ring` bytes (at least two).
template <int PB>
constexpr int scant_stages(int ring) {
    return ring / (scant_gps<PB>() * 4 * (PB + 12)) < 2 ? 2 : ring / (scant_gps<PB>() * 4 * (PB + 12));
}

template <int PB, int NW, int S>
constexpr int scant_smem_bytes() {
    return 65536 + NW * S * (scant_gps<PB>() * 4 * (PB + 12) + 8);
}

template <class U, int NW, int S>
__global__ void __launch_bounds__(NW * 32, 1) scant_kernel(const float *__restrict__ q_rot,
                                                           const float *__restrict__ s_q,
                                                           const float *__restrict__ norms,
                                                           const uint8_t *__restrict__ codes,
                                                           size_t n, float *__restrict__ out,
                                                           Params P, DevTables T) {
    constexpr int PB = U::PB;                // packed bytes per code (trailer offset)
    static_assert(S >= 2, "the ring needs two stages");
    constexpr uint32_t GB = 4u * (PB + 12);  // bytes per group of 4 codes
    constexpr int GPS = scant_gps<PB>();     // groups per stage (a power of two)
    constexpr uint32_t SB = GPS * GB;        // bytes per stage
    constexpr int CW = (PB + 12) / 4;        // words per code
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float s_red[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *tab = smem;
    unsigned char *ring = smem + 65536 + (size_t)warp * S * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 65536 + (size_t)NW * S * SB) + warp * S;
    int *err = T.status;

    // super-group = one stage's GPS groups; warp gw owns super-groups gw, gw + TW, ...
    const size_t SG = n / (4 * GPS);
    const size_t TW = (size_t)gridDim.x * NW;
    const size_t gw = (size_t)blockIdx.x * NW + warp;
    const size_t K = gw < SG ? (SG - gw + TW - 1) / TW : 0;  // super-groups of this warp
    const size_t KG = K * GPS;                               // groups of this warp
    // ring set-up and the first S copies, before the table build
    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(smem_u32(bars + s), 1);
        mbar_init_fence();
        for (int s = 0; s < S && (size_t)s < K; ++s) {
            const uint32_t bar = smem_u32(bars + s);
            mbar_expect_tx(bar, SB);
            bulk_load(smem_u32(ring + s * SB), codes + (gw + (size_t)s * TW) * SB, SB, bar);
        }
    }
    typename U::Query Q;
    int ssum;
    float step;
    U::setup(q_rot, s_q, tab, T, s_red, Q, ssum, step);
    const float qn2 = norms[0], qn = norms[1], sc = P.scale;
    const bool kind0 = !(lane & 4);                               // holds a centroid dot
    const int ec = U::code_of_lane(lane);                         // code of the group

    const size_t src_step = TW * SB;
    const uint8_t *src_next = codes + (gw + (size_t)S * TW) * SB;  // next super-group to fetch
    int s = 0;
    uint32_t ph = 0;
    size_t kg = 0;
    bool ok = true;
    for (size_t k0 = 0; k0 < KG; k0 += 4) {
        // the code this lane finishes: code ec of group ke of this warp
        const size_t ke = k0 + (lane & 3);
        const bool ev = kind0 && ke < KG;
        const size_t ce = 4 * (GPS * (gw + (ke / GPS) * TW) + (ke % GPS)) + ec;
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;  // its trailer, read from the stage below
        float R = 0.0f;
        const int nst = (KG - k0 < 4) ? (int)(KG - k0) : 4;
#pragma unroll 1
        for (int i = 0; i < nst; ++i, ++kg) {
            const int sub = (int)(kg & (GPS - 1));
            const uint32_t bar = smem_u32(bars + s);
            if (sub == 0) {
                ok = __all_sync(kFull, mbar_wait(bar, ph, err, kErrScanWait));
                if (!ok) break;
            }
            const uint32_t *sw = reinterpret_cast<const uint32_t *>(ring + s * SB + sub * GB);
            const float y = U::group([&](int c, int wi) { return sw[c * CW + wi]; }, Q, tab, lane);
            R = ((lane & 3) == i) ? y : R;
            if (kind0 && (lane & 3) == i) {
                // the trailer of the code this lane finishes, from the stage (three
                // conflict-free words for the 4 lanes; from global memory these
                // touched 16 lines per load)
                const float *tw = reinterpret_cast<const float *>(sw + ec * CW) + PB / 4;
                t0 = tw[0];
                t1 = tw[1];
                t2 = tw[2];
            }
            if (sub == GPS - 1) {
                __syncwarp();
                if (lane == 0 && kg / GPS + S < K) {
                    fence_proxy_async_smem();
                    mbar_expect_tx(bar, SB);
                    bulk_load(smem_u32(ring + s * SB), src_next, SB, bar);
                    src_next += src_step;
                }
                if (++s == S) {
                    s = 0;
                    ph ^= 1u;
                }
            }
        }
        if (!ok) break;
        const float sb = __shfl_down_sync(kFull, R, 4);
        if (ev) out[ce] = scan8_distance(R, sb, t0, t1, t2, step, ssum, sc, qn2, qn);
    }
    if (!ok) {
        // wait (bounded) for this warp's copies still in flight, then leave
        if (lane == 0) {
            const size_t k = kg / GPS;
            for (size_t j = k; j < K && j < k + S; ++j) {
                mbar_drain(smem_u32(bars + s), ph);
                if (++s == S) {
                    s = 0;
                    ph ^= 1u;
                }
            }
        }
        return;
    }
    // the last n mod (4 GPS) codes, read straight from global memory by the
    // warp that would own super-group SG, one group at a time
    const size_t c0 = 4 * GPS * SG;
    if (c0 < n && gw == SG % TW) {
        const uint32_t *cw0 = reinterpret_cast<const uint32_t *>(codes);
        for (size_t b = c0; b < n; b += 4) {
            const size_t r = (n - b < 4) ? (n - b) : 4;
            const float y = U::group(
                [&](int c, int wi) {
                    const size_t cc = b + ((size_t)c < r ? (size_t)c : r - 1);
                    return __ldg(cw0 + cc * CW + wi);
                },
                Q, tab, lane);
            const float sb = __shfl_down_sync(kFull, y, 4);
            if (kind0 && (lane & 3) == 0 && (size_t)ec < r) {
                const size_t ce = b + ec;
                const float *tm = reinterpret_cast<const float *>(codes + ce * (PB + 12) + PB);
                out[ce] = scan8_distance(y, sb, __ldg(tm), __ldg(tm + 1), __ldg(tm + 2), step, ssum,
                                         sc, qn2, qn);
            }
        }
    }
}
// Codes whose packed part is narrower than one 32-bit word (D = 4 with
// nibble packing: 2 bytes) are scanned one thread per code with byte loads.
template <bool SYM>
__global__ void __launch_bounds__(256) scan_bytes_kernel(const float *__restrict__ q_rot,
                                                         const float *__restrict__ s_q,
                                                         const float *__restrict__ norms,
                                                         const uint8_t *__restrict__ codes_a,
                                                         const uint8_t *__restrict__ codes, size_t n,
                                                         float *__restrict__ out, size_t ldo,
                                                         Params P, DevTables T) {
    const size_t row = blockIdx.y;
    const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    auto unit = [&](const uint8_t *code, int i) -> unsigned {
        if (P.nibble) {
            const unsigned b = code[i >> 1];
            return (i & 1) ? (b >> 4) : (b & 15u);
        }
        return code[i];
    };
    const uint8_t *code = codes + c * (size_t)P.cs;
    float mb[3];
    for (int q = 0; q < 3; ++q) {
        uint32_t w = 0;
        for (int t = 0; t < 4; ++t) w |= (uint32_t)code[P.pb + 4 * q + t] << (8 * t);
        mb[q] = __uint_as_float(w);
    }
    float d;
    if constexpr (SYM) {
        const uint8_t *ca = codes_a + row * (size_t)P.cs;
        float ma[3];
        for (int q = 0; q < 3; ++q) {
            uint32_t w = 0;
            for (int t = 0; t < 4; ++t) w |= (uint32_t)ca[P.pb + 4 * q + t] << (8 * t);
            ma[q] = __uint_as_float(w);
        }
        float ip = 0.0f;
        for (int i = 0; i < P.D; ++i)
            ip = __fmaf_rn(__fmul_rn(T.centroids[unit(ca, i) >> 1], ma[2]),
                           __fmul_rn(T.centroids[unit(code, i) >> 1], mb[2]), ip);
        const float ipt = __fmul_rn(__fmul_rn(ip, ma[0]), mb[0]);
        d = __fsub_rn(__fadd_rn(__fmul_rn(ma[0], ma[0]), __fmul_rn(mb[0], mb[0])), __fmul_rn(2.0f, ipt));
    } else {
        const float *qr = q_rot + row * (size_t)P.D;
        const float *sq = s_q + row * (size_t)P.D;
        float ip = 0.0f, dot = 0.0f;
        for (int i = 0; i < P.D; ++i) {
            const unsigned u = unit(code, i);
            ip = __fmaf_rn(qr[i], T.centroids[u >> 1], ip);
            dot = __fadd_rn(dot, (u & 1u) ? sq[i] : -sq[i]);
        }
        const float ip_mse = __fmul_rn(ip, mb[2]);
        const float corr = __fmul_rn(__fmul_rn(P.scale, mb[1]), dot);
        const float ipt = __fmul_rn(__fmul_rn(__fadd_rn(ip_mse, corr), mb[0]), norms[2 * row + 1]);
        d = __fsub_rn(__fadd_rn(norms[2 * row], __fmul_rn(mb[0], mb[0])), __fmul_rn(2.0f, ipt));
    }
    out[row * ldo + c] = d > 0.0f ? d : 0.0f;
}

// ---------------------------------------------------------------------------
// Dispatch over log2(D).
// ---------------------------------------------------------------------------
template <template <int> class F, typename... Args>
cudaError_t dispatch_logd(int log2D, Args &&...args) {
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

int sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (count <= 0) count = 148;
    }
    return count;
}

constexpr int kSmemBudget = 227 * 1024;

template <int LOG_D, bool NIBBLE>
cudaError_t encode2_launch(const Params &P, const DevTables &T, const float *X, size_t n,
                           uint8_t *out, cudaStream_t st) {
    constexpr int RPW = enc2_rpw<LOG_D, NIBBLE>();
    const int per_warp = encode2_warp_bytes_c<LOG_D, RPW>();
    int warps = (kSmemBudget - kTabBytes - crep_bytes(P)) / per_warp;
    if (warps > enc2_max_warps<LOG_D, NIBBLE>()) warps = enc2_max_warps<LOG_D, NIBBLE>();
    if (warps < 1) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)kTabBytes + crep_bytes(P) + (size_t)warps * per_warp;
    cudaError_t e = cudaFuncSetAttribute(encode2_kernel<LOG_D, NIBBLE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, encode2_kernel<LOG_D, NIBBLE>, 32 * warps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const size_t groups = (n + RPW - 1) / RPW;
    size_t blocks = (groups + warps - 1) / warps;
    const size_t cap = (size_t)sm_count() * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    encode2_kernel<LOG_D, NIBBLE><<<(unsigned)blocks, 32 * warps, smem, st>>>(X, n, out, P, T);
    return cudaGetLastError();
}

template <int LOG_D>
struct EncodeRun {
    static cudaError_t run(const Params &P, const DevTables &T, const float *X, size_t n,
                           uint8_t *out, cudaStream_t st) {
        if constexpr (LOG_D >= 8 && LOG_D <= 10)
            return P.nibble ? encode2_launch<LOG_D, true>(P, T, X, n, out, st)
                            : encode2_launch<LOG_D, false>(P, T, X, n, out, st);
        constexpr int VPW = LOG_D >= 11 ? 2 : 4;
        auto kern = encode_kernel<LOG_D, VPW>;
        const int D = 1 << LOG_D;
        const int per_warp = encode_warp_bytes(D, P.cs, VPW);
        int warps = (kSmemBudget - kTabBytes) / per_warp;
        if (warps > 8) warps = 8;
        if (warps < 1) return cudaErrorInvalidConfiguration;
        const size_t smem = (size_t)kTabBytes + (size_t)warps * per_warp;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        const size_t groups = (n + VPW - 1) / VPW;
        size_t blocks = (groups + warps - 1) / warps;
        const size_t cap = (size_t)sm_count() * per_sm;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        kern<<<(unsigned)blocks, 32 * warps, smem, st>>>(X, n, out, P, T);
        return cudaGetLastError();
    }
};

template <int LOG_D>
struct PrepareRun {
    static cudaError_t run(const Params &P, const DevTables &T, const float *Q, size_t m,
                           float *q_rot, float *s_q, float *norms, cudaStream_t st) {
        const int D = 1 << LOG_D;
        int warps = (kSmemBudget - kTabBytes) / (4 * (D + 8));
        if (warps > 8) warps = 8;
        if (warps < 1) return cudaErrorInvalidConfiguration;
        const size_t smem = (size_t)kTabBytes + (size_t)warps * 4 * (D + 8);
        cudaError_t e = cudaFuncSetAttribute(prepare_kernel<LOG_D>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        size_t blocks = (m + warps - 1) / warps;
        const size_t cap = (size_t)sm_count() * 4;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        prepare_kernel<LOG_D><<<(unsigned)blocks, 32 * warps, smem, st>>>(Q, m, q_rot, s_q, norms, P, T);
        return cudaGetLastError();
    }
};

template <int LOG_D, bool NIBBLE, bool SYM>
cudaError_t scan_launch(const Params &P, const DevTables &T, const float *q_rot, const float *s_q,
                        const float *norms, const uint8_t *codes_a, size_t m,
                        const uint8_t *codes, size_t n, float *out, size_t ldo, cudaStream_t st) {
    using S = ScanShape<LOG_D, NIBBLE>;
    if constexpr (S::W < 1) {
        const unsigned bx = (unsigned)((n + 255) / 256);
        for (size_t r0 = 0; r0 < m; r0 += 65535) {
            const size_t rows = (m - r0 < 65535) ? (m - r0) : 65535;
            scan_bytes_kernel<SYM><<<dim3(bx, (unsigned)rows), 256, 0, st>>>(
                SYM ? nullptr : q_rot + r0 * (size_t)S::D, SYM ? nullptr : s_q + r0 * (size_t)S::D,
                SYM ? nullptr : norms + 2 * r0, SYM ? codes_a + r0 * (size_t)P.cs : nullptr, codes, n,
                out + r0 * ldo, ldo, P, T);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    } else {
        const int threads = 256;
        const size_t smem = sizeof(float) * ((size_t)(NIBBLE ? 8 : 128) * 32 + (S::QREG ? 0 : 2 * S::PPL * 32));
        auto kern = scan_kernel<LOG_D, NIBBLE, SYM>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        const size_t steps = (n + S::CPS * S::U - 1) / (S::CPS * S::U);
        size_t bx = (steps + (threads / 32) - 1) / (threads / 32);
        size_t cap = (size_t)sm_count() * per_sm;
        // spread the rows over the machine: each row gets its share of CTAs
        if (m > 1) cap = (cap + m - 1) / m;
        if (cap < 1) cap = 1;
        if (bx > cap) bx = cap;
        if (bx < 1) bx = 1;
        for (size_t r0 = 0; r0 < m; r0 += 65535) {
            const size_t rows = (m - r0 < 65535) ? (m - r0) : 65535;
            dim3 grid((unsigned)bx, (unsigned)rows);
            const float *qr = SYM ? nullptr : q_rot + r0 * (size_t)S::D;
            const float *sq = SYM ? nullptr : s_q + r0 * (size_t)S::D;
            const float *nm = SYM ? nullptr : norms + 2 * r0;
            const uint8_t *ca = SYM ? codes_a + r0 * (size_t)P.cs : nullptr;
            kern<<<grid, threads, smem, st>>>(qr, sq, nm, ca, codes, n, out + r0 * ldo, ldo, P, T);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
}

// The staged 1->N scan: one CTA per SM (its shared memory is the centroid
// table plus NW rings), at most as many warps as there are groups of 4 codes.
// 16 warps (4 per scheduler) with ~8 KB rings measured fastest on B200 at
// 10M x 1036-byte codes (12 warps x 3 stages: 80%, 16 x 2: 85% of the copy
// bandwidth; 13 or 14 warps are slower than 12).
template <class U, int NW, int S>
cudaError_t scant_launch(const Params &P, const DevTables &T, const float *q_rot,
                         const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                         float *out, cudaStream_t st) {
    auto kern = scant_kernel<U, NW, S>;
    constexpr int smem = scant_smem_bytes<U::PB, NW, S>();
    static_assert(smem <= kSmemBudget - 64, "scan rings exceed shared memory");
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const size_t groups = n / (4 * scant_gps<U::PB>());
    size_t blocks = (groups + NW - 1) / NW;
    const size_t cap = (size_t)sm_count();
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    kern<<<(unsigned)blocks, NW * 32, smem, st>>>(q_rot, s_q, norms, codes, n, out, P, T);
    return cudaGetLastError();
}

template <int LOG_D>
cudaError_t scan8_launch(const Params &P, const DevTables &T, const float *q_rot, const float *s_q,
                         const float *norms, size_t m, const uint8_t *codes, size_t n, float *out,
                         size_t ldo, cudaStream_t st) {
    if constexpr (LOG_D < 7 || LOG_D > 10) {
        return cudaErrorNotSupported;
    } else {
        constexpr int WPL = (1 << LOG_D) / 128;
        if (m == 1 && (reinterpret_cast<uintptr_t>(codes) & 15) == 0)
            return scant_launch<ByteUnits<WPL>, 16, scant_stages<128 * WPL>(8400)>(
                P, T, q_rot, s_q, norms, codes, n, out, st);
        auto kern = scan8b_kernel<WPL>;
        const int threads = 256;
        const size_t smem = 256 * 256;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        const size_t batches = (n + 15) / 16;
        size_t bx = (batches + (threads / 32) - 1) / (threads / 32);
        size_t cap = (size_t)sm_count() * per_sm;
        if (m > 1) cap = (cap + m - 1) / m;
        if (cap < 1) cap = 1;
        if (bx > cap) bx = cap;
        if (bx < 1) bx = 1;
        for (size_t r0 = 0; r0 < m; r0 += 65535) {
            const size_t rows = (m - r0 < 65535) ? (m - r0) : 65535;
            kern<<<dim3((unsigned)bx, (unsigned)rows), threads, smem, st>>>(
                q_rot + r0 * (size_t)(1 << LOG_D), s_q + r0 * (size_t)(1 << LOG_D), norms + 2 * r0,
                codes, n, out + r0 * ldo, ldo, P, T);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
}

// The staged 1->N scan of nibble codes: D = 128 with a half-warp per code,
// D = 256 .. 2048 with WPL = D / 256 words per lane (D = 2048 needs more query
// registers, so 12 warps).
template <int LOG_D>
cudaError_t scan4t_launch(const Params &P, const DevTables &T, const float *q_rot,
                          const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                          float *out, cudaStream_t st) {
    if constexpr (LOG_D < 7 || LOG_D > 11) {
        return cudaErrorNotSupported;
    } else if constexpr (LOG_D == 7) {
        return scant_launch<HalfNibbleUnits, 16, scant_stages<64>(8400)>(P, T, q_rot, s_q, norms, codes, n,
                                                                 out, st);
    } else {
        constexpr int WPL = (1 << LOG_D) / 256;
        if constexpr (WPL <= 4)
            return scant_launch<NibbleUnits<WPL>, 16, scant_stages<128 * WPL>(8400)>(P, T, q_rot, s_q, norms, codes, n,
                                                                 out, st);
        else
            return scant_launch<NibbleUnits<WPL>, 12, scant_stages<128 * WPL>(12600)>(P, T, q_rot, s_q, norms, codes,
                                                                  n, out, st);
    }
}

template <int LOG_D>
struct ScanRun {
    static cudaError_t run(const Params &P, const DevTables &T, const float *q_rot,
                           const float *s_q, const float *norms, const uint8_t *codes_a, size_t m,
                           const uint8_t *codes, size_t n, float *out, size_t ldo, bool sym,
                           cudaStream_t st) {
        if (!P.nibble && !sym && LOG_D >= 7 && LOG_D <= 10)
            return scan8_launch<LOG_D>(P, T, q_rot, s_q, norms, m, codes, n, out, ldo, st);
        if (P.nibble && !sym && m == 1 && LOG_D >= 7 && LOG_D <= 11 &&
            (reinterpret_cast<uintptr_t>(codes) & 15) == 0)
            return scan4t_launch<LOG_D>(P, T, q_rot, s_q, norms, codes, n, out, st);
        if (P.nibble) {
            return sym ? scan_launch<LOG_D, true, true>(P, T, q_rot, s_q, norms, codes_a, m, codes,
                                                        n, out, ldo, st)
                       : scan_launch<LOG_D, true, false>(P, T, q_rot, s_q, norms, codes_a, m,
                                                         codes, n, out, ldo, st);
        }
        return sym ? scan_launch<LOG_D, false, true>(P, T, q_rot, s_q, norms, codes_a, m, codes, n,
                                                     out, ldo, st)
                   : scan_launch<LOG_D, false, false>(P, T, q_rot, s_q, norms, codes_a, m, codes,
                                                      n, out, ldo, st);
    }
};

}  // namespace

cudaError_t launch_encode(const Params &P, const DevTables &T, const float *X, size_t n,
                          uint8_t *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    return dispatch_logd<EncodeRun>(P.log2D, P, T, X, n, out, st);
}

cudaError_t launch_prepare(const Params &P, const DevTables &T, const float *Q, size_t m,
                           float *q_rot, float *s_q, float *norms, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    return dispatch_logd<PrepareRun>(P.log2D, P, T, Q, m, q_rot, s_q, norms, st);
}

cudaError_t launch_scan_1_to_n(const Params &P, const DevTables &T, const float *q_rot,
                               const float *s_q, const float *norms, const uint8_t *codes,
                               size_t n, float *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    return dispatch_logd<ScanRun>(P.log2D, P, T, q_rot, s_q, norms, (const uint8_t *)nullptr,
                                  (size_t)1, codes, n, out, n, false, st);
}

cudaError_t launch_mton_fp32(const Params &P, const DevTables &T, const float *q_rot,
                             const float *s_q, const float *norms, size_t m,
                             const uint8_t *codes, size_t n, float *out, size_t ldo,
                             cudaStream_t st) {
    if (n == 0 || m == 0) return cudaSuccess;
    return dispatch_logd<ScanRun>(P.log2D, P, T, q_rot, s_q, norms, (const uint8_t *)nullptr, m,
                                  codes, n, out, ldo, false, st);
}

cudaError_t launch_mton_sym_fp32(const Params &P, const DevTables &T, const uint8_t *A,
                                 size_t m, const uint8_t *B, size_t n, float *out, size_t ldo,
                                 cudaStream_t st) {
    if (n == 0 || m == 0) return cudaSuccess;
    return dispatch_logd<ScanRun>(P.log2D, P, T, (const float *)nullptr, (const float *)nullptr,
                                  (const float *)nullptr, A, m, B, n, out, ldo, true, st);
}

}  // namespace tq
