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

// Counters of the exact stages (device ints, zeroed before each batch): rows
// the certificate left open, candidates outside the bound, open rows taken by
// the exact scan, and rows taken by the list pass (see launch_fallback).
enum {
    kCntFallbackRows = 0,
    kCntBoundViolations = 1,
    kCntScanRows = 2,
    kCntListRows = 3,
    kCntWords = 4
};

// Codes collected per open row by a threshold pass.
constexpr int kCollectCap = 1024;
// The tensor-core threshold pass runs when more rows than this are open (one
// pass over the corpus for up to 128 rows costs about what the exact scan
// costs for five).
constexpr int kTensorTierMinRows = 4;

// Candidate rescoring: one warp per query row (row count read from m_dev).
// cand_d / cand_i hold each row's kc (<= 32) tensor-pass candidates, ascending
// by (approximate distance, index), index -1 past the corpus.  Each candidate
// is rescored with the reference's own arithmetic; the row's k best by
// (distance, index) go to out_d / out_i.  The row is certified when its k-th
// exact distance is below the kc-th approximate distance minus the error
// bound of the tensor pass (so no code outside the candidates can enter the
// top-k); otherwise its index is appended to fail_rows (counters[0]), its k-th
// exact candidate distance e_k to thr and e_k + eps (rounded up; -1 when a
// candidate broke the bound) to tthr, at the same position.  A candidate whose
// approximate and exact distances differ by more than the bound eps is counted
// in counters[1] and fails its row as well.
// cmax = max_v |c_v| of the space's centroid table; kappa = the tensor pass's
// relative error bound (tc_topk_kappa of the variant that produced the
// candidates); kappa_t = that of the threshold pass over open rows (tthr is
// e_k plus the bound with max(kappa, kappa_t)).
cudaError_t launch_rescore(const Params &P, const float *centroids, float cmax, const int *m_dev,
                           int kc, int k, const float *cand_d, const long long *cand_i,
                           const float *q_rot, const float *s_q, const float *norms,
                           const uint8_t *codes, size_t n, const float *bound, float kappa,
                           float kappa_t, float bound_scale,
                           float *out_d, long long *out_i, int *fail_rows, float *thr, float *tthr,
                           int *counters, int max_rows, cudaStream_t st);

// The open rows' query planes and scales, gathered to rows 0 .. nf-1 for the
// tensor-core threshold pass (nothing unless nf = counters[0] exceeds
// kTensorTierMinRows).  Planes: rows of K BF16 values.
cudaError_t launch_gather_open(const int *counters, const int *fail_rows, const void *ah,
                               const void *al, const float *r1, const float *r2, int K,
                               int max_rows, void *ah2, void *al2, float *r1o, float *r2o,
                               cudaStream_t st);

// Device buffers of the fallback (R = max_rows open rows at most).
struct FallbackBuffers {
    const float *thr;   // R: e_k, from the rescoring
    const float *tthr;  // R: e_k + eps, from the rescoring
    int *coll_n;        // 2R: counts of the tensor pass's lists, then of the exact scan's
    float *coll_d;      // R * kCollectCap
    int *coll_i;        // R * kCollectCap: the tensor pass's lists, then the exact scan's
    int *scan_rows;     // R: positions in fail_rows taken by the exact scan
    int *list_rows;     // R: rows taken by the list pass
    float *part_d;      // R * fb_ctas * k
    int *part_i;        // R * fb_ctas * k
};

// The rows in fail_rows, exact by construction, in three tiers:
//   1. (tensor_pass: launch_tc_thresh ran on the gathered open rows with
//      thr = tthr, lists in coll_i / coll_n[0..R)) when more than
//      kTensorTierMinRows rows are open and the row's bound held: the k best
//      of its list by (exact distance, index).  Every code of the true top-k
//      is in the list: its tensor-pass distance is at most its exact one +
//      eps <= e_k + eps.
//   2. the others: an exact scan of every code, collecting those at or below
//      e_k (every member of the true top-k), then the k best of them.
//   3. rows with more than kCollectCap codes in tier 2: a full pass with
//      per-CTA top-k lists (fb_ctas CTAs) merged per row.
// Every kernel returns at once when it has no row.
int fallback_ctas(int sms);
cudaError_t launch_fallback(const Params &P, const float *centroids, int k, const float *q_rot,
                            const float *s_q, const float *norms, const uint8_t *codes, size_t n,
                            const int *fail_rows, int *counters, int fb_ctas, bool tensor_pass,
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
// The reference-order symmetric distances of m codes A against n codes B,
// out[i * ldo + j]: one thread per pair (distBuildAVX / distBuildScalarB4 as
// the reference's Release build evaluates them).
cudaError_t launch_exact_mton_sym(const Params &P, const float *centroids, const uint8_t *A, size_t m,
                                  const uint8_t *B, size_t n, float *out, size_t ldo, cudaStream_t st);

}  // namespace tq
