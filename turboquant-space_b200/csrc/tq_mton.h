// tq_mton.h -- operand planes and contraction kernels of the M x N distances
// (tq_mton.cu: decode + FP32 SGEMM; tq_tc.cu: split-BF16 tcgen05 GEMM).
#pragma once

#include "tq_internal.h"

namespace tq {

constexpr int kPlaneF32 = 0;   // one FP32 plane
constexpr int kPlaneBF16 = 1;  // hi and lo BF16 planes, x = hi + lo
constexpr int kPlaneRowAlign = 128;

// Columns of the BF16 lo plane of asymmetric code planes: the QJL half of
// those planes is exact (+-1, see tq_mton.cu), so lo is stored for the
// centroid half only, rounded up to a whole 64-wide K block.
inline int asym_lo_width(int D) { return D % 64 == 0 ? D : 2 * D; }

// Rows [0, rows) of `codes` -> planes of rows_pad x K (K = D symmetric, 2D
// asymmetric), zero rows beyond `rows`; s1/s2 per-row scalars (rows_pad).
// BF16 lo planes have K columns, asym_lo_width(D) for asymmetric planes.
cudaError_t launch_planes_from_codes(const Params &P, const DevTables &T, const uint8_t *codes,
                                     size_t rows, size_t rows_pad, bool sym, int fmt, void *plane0,
                                     void *plane1, float *s1, float *s2, cudaStream_t st);

// Prepared queries -> planes of rows_pad x 2D and r1 = |q|, r2 = |q|^2.
cudaError_t launch_planes_from_prepared(const float *q_rot, const float *s_q, const float *norms,
                                        size_t rows, size_t rows_pad, int D, int fmt, void *plane0,
                                        void *plane1, float *r1, float *r2, cudaStream_t st);

// out[i, j] = max(0, r2_i + c2_j - 2 (C_ij r1_i) c1_j), C = A B^T in FP32.
cudaError_t launch_sgemm_dist(const float *A, const float *B, int K, size_t m, size_t m_pad,
                              size_t n, size_t n_pad, const float *r1, const float *r2,
                              const float *c1, const float *c2, float *out, size_t ldo,
                              cudaStream_t st);

// The same with C = Ah Bh^T + Ah Bl^T + Al Bh^T on tcgen05 tensor cores
// (FP32 accumulators in tensor memory, promoted to an IEEE FP32 running sum
// every few K blocks).  K % 64 == 0, m_pad % 128 == 0, n_pad % 128 == 0.  Bl has k_lo columns (k_lo % 64 == 0, k_lo <= K): B's lo
// part is zero beyond them, where the Ah Bl^T product is skipped.  `err`
// (device int) is set non-zero if a bounded wait in the kernel gave up.
cudaError_t launch_tc_dist(const void *Ah, const void *Al, const void *Bh, const void *Bl, int K,
                           int k_lo, size_t m, size_t m_pad, size_t n, size_t n_pad, const float *r1,
                           const float *r2, const float *c1, const float *c2, float *out,
                           size_t ldo, int *err, cudaStream_t st);

// Top-k over a device-resident index: C = A B^T as above, reduced per row to the
// k (<= kCandMax) smallest (distance, index) pairs, ties to the smaller index.
// The row count is read from m_dev; `grid` CTAs split the rows into 128-row
// blocks and the columns into slices.
// Variants 0 and 5: 128 x 256 tiles (n_pad % 256 == 0), two partial lists per
// (row, slice); 1-4: 128 x 128 tiles (tc_topk_shape gives each one's stages
// and chunk length).  The partial buffers
// hold grid * 128 * tc_topk_lists(variant) * kCandMax entries.
// The column operand of the decoded-B tensor kernels: instead of BF16 planes,
// four decoder warps per CTA write each K block's B tile into shared memory
// straight from the codes (a centroid block as the hi/lo pair of the table
// value c[idx], a sign block as the exact +-1), and the per-code scale of the
// asymmetric form is applied per column when a chunk is promoted: fc for the
// centroid half (sigma / (scale gamma), or sigma), fs for the sign half (1, or
// 0 for a code whose sign half is left out), as launch_dec_factors computes
// them; c1 / c2 of the epilogue come from the same kernel.
struct DecSrc {
    const uint8_t *codes = nullptr;      // column codes, cs bytes apart, 16-byte aligned base,
                                         // readable up to 15 bytes past the last code
    unsigned n = 0;                      // columns; tile columns at or past n decode to zero
    int cs = 0;                          // code bytes (a multiple of 4)
    int nibble = 0;                      // two units per byte (bits <= 4)
    int kbc = 0;                         // K blocks (64 values) of the centroid half
    const float *fc = nullptr, *fs = nullptr;  // per-column factors (asymmetric); null: none
    const float *centroids = nullptr;    // the space's centroid table (device)
    int levels = 0;
    // set by the launcher: shared-memory buffers of one tile of codes (128 codes,
    // one bulk copy each) and their size
    int cbufs = 0, ctile_bytes = 0;
};

// Per-code scalars of the decoded-B kernels for rows [0, rows) of `codes`
// (zero for rows up to rows_pad): asymmetric: c1 = scale gamma |x| (or |x|),
// c2 = |x|^2, fc, fs as above; symmetric: c1 = sigma |x|, c2 = |x|^2 (fc, fs
// may be null).
cudaError_t launch_dec_factors(const Params &P, const uint8_t *codes, size_t rows, size_t rows_pad,
                               bool sym, float *c1, float *c2, float *fc, float *fs, cudaStream_t st);

constexpr int kTopKMax = 16;   // results per row (k) of the serving path
constexpr int kCandMax = 32;   // list length of the tensor-core top-k (candidates per row)
constexpr int kTopKListsMax = 2;
int tc_topk_variants();
// Relative error bound of a variant's tensor pass (see the exact stage's
// certificate), for K columns of which the first k_lo have a lo plane.
float tc_topk_kappa(int variant, int K, int k_lo);
int tc_topk_lists(int variant);
// {rows per CTA, codes per tile, pipeline stages, K blocks per chunk} of a variant
bool tc_topk_shape(int variant, int out[4]);
cudaError_t launch_tc_topk(int variant, const void *Ah, const void *Al, size_t rows_pad,
                           const void *Bh, const void *Bl, size_t n_pad, int K, int k_lo,
                           const int *m_dev,
                           size_t n, const float *r1, const float *r2, const float *c1,
                           const float *c2, int k, float *part_d, int *part_i,
                           unsigned long long *gthr, int *err, int grid, cudaStream_t st);
// The same top-k with decoded B tiles (variants 1-4, the 128 x 128 tiles; no
// planes of the columns).  K = 2D; dec.kbc = D / 64.
cudaError_t launch_tc_topk_dec(int variant, const void *Ah, const void *Al, size_t rows_pad,
                               const DecSrc &dec, size_t n_pad, int K, const int *m_dev, size_t n,
                               const float *r1, const float *r2, const float *c1, const float *c2,
                               int k, float *part_d, int *part_i, unsigned long long *gthr, int *err,
                               int grid, cudaStream_t st);
// Whether `variant` runs with decoded B tiles for codes of cs bytes (a tile of
// 128 codes must fit in shared memory beside the variant's stages).
bool tc_topk_dec_ok(int variant, int cs);
// The M x N distances of launch_tc_dist with decoded B tiles (128 x 128 tiles,
// two stages): columns [0, dec.n) of dec.codes, out[i * ldo + j] for i < m.
// Asymmetric (dec.fc, dec.fs set): K = 2D, dec.kbc = D / 64, c1 / c2 / fc / fs
// from launch_dec_factors; symmetric (dec.fc null): K = D, dec.kbc = D / 64,
// A the symmetric row planes.  The last tile's copy reads the codes up to a
// 16-byte boundary past code dec.n - 1: the caller guarantees that memory.
cudaError_t launch_tc_dist_dec(const void *Ah, const void *Al, size_t m, size_t m_pad, const DecSrc &dec,
                               size_t n_pad, int K, const float *r1, const float *r2, const float *c1,
                               const float *c2, float *out, size_t ldo, int *err, cudaStream_t st);
// Whether a tile of 128 codes of cs bytes fits launch_tc_dist_dec's shared memory.
bool tc_dist_dec_fits(int cs);
// Threshold collection over the corpus for the rows of A (row count *m_dev,
// nothing unless it exceeds min_rows): every column whose tile distance (as the
// top-k pass computes it) is at most thr[row] goes to coll_i[row * cap + ...],
// counted in coll_n[row] (which may exceed cap: overflow).  Planes (Bh, Bl,
// k_lo) or, with dec, decoded B tiles: the tile shape of variant
// tc_thresh_variant(dec != nullptr, n_pad) (6 on planes, 4 decoded), whose
// error bound (tc_topk_kappa) the thresholds must allow for.
int tc_thresh_variant(bool decoded, size_t n_pad);
cudaError_t launch_tc_thresh(const void *Ah, const void *Al, size_t rows_pad, const void *Bh,
                             const void *Bl, const DecSrc *dec, size_t n_pad, int K, int k_lo,
                             const int *m_dev, int min_rows, size_t n, const float *r1,
                             const float *r2, const float *c1, const float *c2, const float *thr,
                             int *coll_n, int *coll_i, int cap, int *err, int grid, cudaStream_t st);
cudaError_t launch_topk_merge(const int *m_dev, int grid_ctas, int lists, const float *part_d,
                              const int *part_i, int k, size_t max_rows, float *out_d,
                              long long *out_i, cudaStream_t st);

// The two contractions of the QJL-corrected symmetric distances on tcgen05
// tensor cores: C1 = A1 B1^T (K1) and C2 = A2 B2^T (K2) over hi/lo TF32 planes
// (FP32 containers, launch_symq_planes_tf32), then out[i, j] = max(0, na^2 + nb^2 -
// 2 (C1 s1a s1b + clamp(C2 s2a s2b, +-|C1 s1a s1b|)) na nb) with the 8-float
// row scalars sa / sb of tq_symq.cu.  exact2: both K2 planes are +-1 (lo
// zero), one product per K step there.  K1, K2 % 32 == 0, m_pad % 128 == 0,
// n_pad % 256 == 0.
cudaError_t launch_tc_symq(const void *A1h, const void *A1l, const void *B1h, const void *B1l,
                           int K1, const void *A2h, const void *A2l, const void *B2h,
                           const void *B2l, int K2, bool exact2, size_t m, size_t m_pad, size_t n,
                           size_t n_pad, const float *sa, const float *sb, float *out, size_t ldo,
                           int *err, cudaStream_t st);

// One thread waits on an mbarrier nothing arrives at; after budget_cycles the
// wait gives up and writes a non-zero code to *err (the failure path of every
// bounded wait in the tensor-core kernels).
cudaError_t launch_bounded_wait_selftest(int *err, long long budget_cycles, cudaStream_t st);

}  // namespace tq
