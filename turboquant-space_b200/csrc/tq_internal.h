// tq_internal.h -- shared declarations of the B200 TurboQuant library
// (host side tq_space.cpp / tq_capi.cu and device side tq_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace tq {

// Largest padded dimension the kernels are instantiated for (log2).
constexpr int kMinLogD = 2;   // D = 4 (the reference pads dim < 4 up to 4)
constexpr int kMaxLogD = 13;  // D = 8192
constexpr int kMaxLevels = 256;
constexpr int kQlutBuckets = 2048;  // bucket table of the b >= 6 quantizer
constexpr int kQlutMaxK = 4;        // boundaries checked per bucket (upper bound)

// Constants the reference's pinned Release build folded into encodeVector
// (space_turbo_quant.h:348, 357-359) and prepareQuery (:447):
//   `norm > 1e-10f` compiles to `norm_sq > fl(1e-10f * 1e-10f)`,
//   the sigma floor is 1e-10f and its inverse fl(1 / 1e-10f).
constexpr uint32_t kNormSqFloorBits = 0x1E3CE509u;
constexpr uint32_t kSigmaFloorBits = 0x2EDBE6FFu;
constexpr uint32_t kInvSigmaFloorBits = 0x501502F9u;

// Geometry and per-space scalars, passed by value to every kernel.
struct Params {
    int dim;           // input dimension
    int D;             // padded power-of-two dimension
    int log2D;
    int bits;          // bits_per_coord (2..9)
    int nibble;        // bits <= 4: two units per byte
    int levels;        // 2^(bits-1) centroids
    int nb;            // levels - 1 boundaries
    int pb;            // packed bytes
    int cs;            // code size = pb + 12
    int lutq;          // 1: quantize through the bucket table (nb > 15)
    int qlut_k;        // boundaries compared per bucket
    int qflag;         // 1: T.qlutf holds lo | 0x80 for the buckets that hold a boundary
                       //    (levels <= 128, qlut_k = 1)
    float qlut_s;      // bucket(v) = clamp(fma(v, qlut_s, qlut_c), 0, NB-1)
    float qlut_c;
    float scale;       // sqrt(pi/2)/sqrt(D)            space_turbo_quant.h:265
    float wht_scale;   // 1/sqrt(D)                     turbo_quant.h:69
};

// Device copies of the space's tables (one allocation per space).
struct DevTables {
    const float *centroids;   // [levels]
    const float *boundaries;  // [nb + kQlutMaxK], padded with +inf
    const uint8_t *qlut;      // [kQlutBuckets]: boundaries below the bucket
    const uint8_t *qlutf;     // [kQlutBuckets]: the same | 0x80 when a boundary lies in the
                              // bucket (P.qflag); otherwise a copy of qlut
    const uint32_t *rot_mask; // [D/32 rounded up]: bit i set <=> rot sign +1
    const uint32_t *qjl_mask; // [D/32 rounded up]
    int *status;              // stream-ordered kernels' error word (0 = ok)
};

// ---- kernel launchers (tq_kernels.cu); all stream-ordered -------------------
cudaError_t launch_encode(const Params &P, const DevTables &T, const float *X, size_t n,
                          uint8_t *out, cudaStream_t st);
cudaError_t launch_prepare(const Params &P, const DevTables &T, const float *Q, size_t m,
                           float *q_rot, float *s_q, float *norms, cudaStream_t st);
cudaError_t launch_scan_1_to_n(const Params &P, const DevTables &T, const float *q_rot,
                               const float *s_q, const float *norms, const uint8_t *codes,
                               size_t n, float *out, cudaStream_t st);
cudaError_t launch_mton_fp32(const Params &P, const DevTables &T, const float *q_rot,
                             const float *s_q, const float *norms, size_t m,
                             const uint8_t *codes, size_t n, float *out, size_t ldo,
                             cudaStream_t st);
cudaError_t launch_mton_sym_fp32(const Params &P, const DevTables &T, const uint8_t *A,
                                 size_t m, const uint8_t *B, size_t n, float *out, size_t ldo,
                                 cudaStream_t st);

// ---- rotated coordinates and QJL-corrected symmetric distances (tq_symq.cu)
cudaError_t launch_rotated_coords(const Params &P, const DevTables &T, const float *X, size_t n,
                                  float *out, cudaStream_t st);
// Plane modes: the three distance variants and the prepared-code export
// (P1 = recon, P2 = signs).
enum SymqMode { SYMQ_LIGHT = 0, SYMQ_FULL = 1, SYMQ_FULL_PREPARED = 2, SYMQ_PREPARE = 3 };
int symq_ldk(int K);            // K rounded up to the GEMM's K step
int symq_k2(int mode, int D);   // columns of the correction plane
cudaError_t launch_symq_planes(const Params &P, const DevTables &T, const uint8_t *codes,
                               size_t rows, int mode, bool row_side, float *P1, int ldk1,
                               float *P2, int ldk2, float *scal, cudaStream_t st);
// The same planes as hi/lo TF32 pairs in FP32 containers (hi = tf32(v),
// lo = tf32(v - hi)): H1/L1 rows_pad x K1, H2/L2 rows_pad x K2, zero past the
// planes' columns and past `rows`; L2 may be null for the light variant
// (exact +-1 signs, lo = 0).  Scalars for the first `rows` rows.
cudaError_t launch_symq_planes_tf32(const Params &P, const DevTables &T, const uint8_t *codes,
                                    size_t rows, size_t rows_pad, int mode, bool row_side,
                                    float *H1, float *L1, int K1, float *H2, float *L2, int K2,
                                    float *scal, cudaStream_t st);
cudaError_t launch_symq_prepared_row(const float *recon, const float *sign, const float *sc, int D,
                                     float *P1, int ldk1, float *P2, int ldk2, float *scal,
                                     cudaStream_t st);
cudaError_t launch_symq_gemm(const float *P1a, const float *P2a, const float *sa, size_t m,
                             const float *P1b, const float *P2b, const float *sb, size_t n,
                             int ldk1, int ldk2, float *out, size_t ldo, cudaStream_t st);

}  // namespace tq
