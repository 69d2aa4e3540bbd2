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

// Counters of the exact stages (device ints, zeroed before each batch):
// rows the certificate left open, candidates outside the bound, and open rows
// whose collection overflowed (answered by the list pass).
enum { kCntFallbackRows = 0, kCntBoundViolations = 1, kCntOverflowRows = 2, kCntWords = 4 };

// Codes collected per open row by the fallback's threshold pass.
constexpr int kCollectCap = 1024;

// Candidate rescoring: one warp per query row (row count read from m_dev).
// cand_d / cand_i hold each row's kc (<= 32) tensor-pass candidates, ascending
// by (approximate distance, index), index -1 past the corpus.  Each candidate
// is rescored with the reference's own arithmetic; the row's k best by
// (distance, index) go to out_d / out_i.  The row is certified when its k-th
// exact distance is below the kc-th approximate distance minus the error
// bound of the tensor pass (so no code outside the candidates can enter the
// top-k); otherwise its index is appended to fail_rows (counters[0]) and its
// k-th exact candidate distance to thr at the same position.  A candidate
// whose approximate and exact distances differ by more than the bound is
// counted in counters[1] and fails its row as well.
// cmax = max_v |c_v| of the space's centroid table.
cudaError_t launch_rescore(const Params &P, const float *centroids, float cmax, const int *m_dev,
                           int kc, int k, const float *cand_d, const long long *cand_i,
                           const float *q_rot, const float *s_q, const float *norms,
                           const uint8_t *codes, size_t n, const float *bound, float bound_scale,
                           float *out_d, long long *out_i, int *fail_rows, float *thr,
                           int *counters, int max_rows, cudaStream_t st);

// Device buffers of the fallback (max_rows = R open rows at most).
struct FallbackBuffers {
    const float *thr;  // R: written by the rescoring
    int *coll_n;       // R
    float *coll_d;     // R * kCollectCap
    int *coll_i;       // R * kCollectCap
    int *fail2;        // R: rows whose collection overflowed
    float *part_d;     // R * fb_ctas * k
    int *part_i;       // R * fb_ctas * k
};

// Fallback for the rows in fail_rows, exact by construction:
//   collect  every code whose exact distance is at most the row's thr (the
//            k-th exact distance among its candidates, so at least the true
//            k-th: every member of the true top-k passes);
//   select   the k best collected by (distance, index) into out_d / out_i;
//   a row that collected more than kCollectCap codes goes to a full pass
//   with per-CTA top-k lists (fb_ctas CTAs) merged per row.
// Every kernel returns at once when it has no row.
int fallback_ctas(int sms);
cudaError_t launch_fallback(const Params &P, const float *centroids, int k, const float *q_rot,
                            const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                            const int *fail_rows, int *counters, int fb_ctas,
                            const FallbackBuffers &fb, float *out_d, long long *out_i,
                            int max_rows, cudaStream_t st);

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
