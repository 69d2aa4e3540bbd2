// tq_exact.h -- the reference's asymmetric distance in the reference build's
// own summation order on the GPU (tq_exact.cu), and the serving path's exact
// top-k stages built on it.
#pragma once

#include "tq_internal.h"

namespace tq {

// Index-wide constants of the certificate's error bound (tq_exact.cu):
// bound[0] = max_j sigma_j |x_j|, bound[1] = max_j scale gamma_j |x_j|,
// bound[2] = max_j |x_j|^2, bound[3] = max_j |x_j|.
constexpr int kBoundFloats = 4;
cudaError_t launch_index_bound(const Params &P, const uint8_t *codes, size_t n, float *bound,
                               cudaStream_t st);

// Counters of the exact stages (device ints, zeroed before each batch).
enum { kCntFallbackRows = 0, kCntBoundViolations = 1, kCntWords = 4 };

// Candidate rescoring: one warp per query row (row count read from m_dev).
// cand_d / cand_i hold each row's kc (<= 32) tensor-pass candidates, ascending
// by (approximate distance, index), index -1 past the corpus.  Each candidate
// is rescored with the reference's own arithmetic; the row's k best by
// (distance, index) go to out_d / out_i.  The row is certified when its k-th
// exact distance is below the kc-th approximate distance minus the error
// bound of the tensor pass (so no code outside the candidates can enter the
// top-k); otherwise its index is appended to fail_rows (counters[0]).  A
// candidate whose approximate and exact distances differ by more than the
// bound is counted in counters[1] and fails its row as well.
// cmax = max_v |c_v| of the space's centroid table.
cudaError_t launch_rescore(const Params &P, const float *centroids, float cmax, const int *m_dev,
                           int kc, int k, const float *cand_d, const long long *cand_i,
                           const float *q_rot, const float *s_q, const float *norms,
                           const uint8_t *codes, size_t n, const float *bound, float bound_scale,
                           float *out_d, long long *out_i, int *fail_rows, int *counters,
                           int max_rows, cudaStream_t st);

// Fallback for the rows in fail_rows: the exact distances of every code with a
// per-CTA top-k (fb_ctas CTAs), merged per row into out_d / out_i.  Both
// kernels return at once when counters[0] is zero.  part_d / part_i hold
// max_rows * fb_ctas * k entries.
int fallback_ctas(int sms);
cudaError_t launch_fallback(const Params &P, const float *centroids, int k, const float *q_rot,
                            const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                            const int *fail_rows, const int *counters, int fb_ctas, float *part_d,
                            int *part_i, float *out_d, long long *out_i, int max_rows,
                            cudaStream_t st);

// Serving admission pool -> batch: out[r] = pool[rows[r]] (dim floats each)
// for r < *m_dev (at most max_rows).
cudaError_t launch_gather_rows(const float *pool, const int *rows, const int *m_dev, size_t dim,
                               size_t max_rows, float *out, cudaStream_t st);

// The reference-order distances of m prepared queries against n codes,
// out[i * ldo + j]: one thread per pair, the arithmetic the rescoring uses.
cudaError_t launch_exact_mton(const Params &P, const float *centroids, const float *q_rot,
                              const float *s_q, const float *norms, size_t m, const uint8_t *codes,
                              size_t n, float *out, size_t ldo, cudaStream_t st);

}  // namespace tq
