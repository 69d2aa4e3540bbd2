/*
 * tq_oracle.h -- plain-C restatement of TurboQuant's encode-and-scan path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the CPU checker the CUDA path is compared
 * against; the product (libtqb200.so and the turboquant Python package) never
 * links, loads or calls it.
 *
 * It restates, step by step, the reference header-only library
 * (include/turboquant/turbo_quant.h, include/turboquant/space_turbo_quant.h)
 * as compiled by the reference's portable Release build
 * (-O3 -ffast-math -fno-finite-math-only -march=x86-64-v3).  Every rounding
 * step of that build is written out explicitly (the 8-lane reduction trees,
 * the FMA contractions, the comparison constants the compiler folded), so that
 * the encode reproduces the reference's code bytes, trailer floats included.
 *
 * Parity: pinned against the reference itself compiled here from its own
 * sources (oracle/Makefile, target `ref`) -- see tests/test_oracle_pin.py and
 * the committed golden vectors under tests/golden/.
 */
#ifndef TQ_ORACLE_H
#define TQ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tqo_space tqo_space;

/* splitmix64 sign vector: turbo_quant.h:27-39, 74-86. */
void tqo_signs(size_t d, uint64_t seed, float *out);

/* Gaussian Lloyd-Max table for `bits` MSE bits: space_turbo_quant.h:76-131.
 * Writes 2^bits centroids and 2^bits - 1 ascending boundaries. */
void tqo_lloyd_max(int bits, float *centroids, float *boundaries);

/* Geometry: space_turbo_quant.h:233-238, 258-266; turbo_quant.h:177-184. */
size_t tqo_padded_dim(size_t dim);
size_t tqo_packed_bytes(size_t padded_dim, int bits_per_coord);
size_t tqo_code_size(size_t padded_dim, int bits_per_coord);

tqo_space *tqo_create(size_t dim, int bits_per_coord, uint64_t rot_seed,
                      uint64_t qjl_seed);
void tqo_destroy(tqo_space *sp);
size_t tqo_space_padded_dim(const tqo_space *sp);
size_t tqo_space_code_size(const tqo_space *sp);
float tqo_space_scale(const tqo_space *sp);
const float *tqo_space_centroids(const tqo_space *sp);
const float *tqo_space_boundaries(const tqo_space *sp);
const float *tqo_space_rot_signs(const tqo_space *sp);
const float *tqo_space_qjl_signs(const tqo_space *sp);

/* The reference's FP32 sum-of-squares reduction tree as its pinned build
 * compiles it (space_turbo_quant.h:343-344, 354-355, 370-371). */
float tqo_sq_reduce(const float *x, size_t n);

/* encodeVector / encodeBatch: space_turbo_quant.h:339-407 (bit-exact). */
void tqo_encode_batch(const tqo_space *sp, const float *X, size_t n,
                      uint8_t *out, int num_threads);

/* prepareQuery: space_turbo_quant.h:439-460.  norms[0] = |q|^2, norms[1] = |q|. */
void tqo_prepare_query(const tqo_space *sp, const float *q, float *q_rot,
                       float *s_q, float *norms);

/* FP32 distances with the reference formulas (space_turbo_quant.h:659-714,
 * 951-1019) and its batch drivers (:577-615). Output row-major [m, n]. */
void tqo_distance_1_to_n(const tqo_space *sp, const float *q,
                         const uint8_t *codes, size_t n, float *out,
                         int num_threads);
void tqo_distance_m_to_n(const tqo_space *sp, const float *Q, size_t m,
                         const uint8_t *codes, size_t n, float *out,
                         int num_threads);
void tqo_distance_m_to_n_symmetric(const tqo_space *sp, const uint8_t *A,
                                   size_t m, const uint8_t *B, size_t n,
                                   float *out, int num_threads);

/* The same formulas evaluated in FP64 on the same codes and the same FP32
 * query (the query preparation itself is redone in FP64). */
double tqo_distance_f64(const tqo_space *sp, const float *q,
                        const uint8_t *code);
double tqo_distance_symmetric_f64(const tqo_space *sp, const uint8_t *a,
                                  const uint8_t *b);

/* rotatedCoordsBatch: space_turbo_quant.h:411-435.  out is [n, padded_dim]. */
void tqo_rotated_coords_batch(const tqo_space *sp, const float *X, size_t n, float *out,
                              int num_threads);

/* QJL-corrected symmetric distances (space_turbo_quant.h:483-572, 731-945):
 * LIGHT adds the sign-agreement term only, FULL all four inner-product terms
 * (two reconstructions + QJL Hadamards per pair), FULL_PREPARED prepares the
 * row code once (prepareSymmetricQuery :499-535) and uses the post-Hadamard
 * dot as the MSE term.  The correction is clamped to +-|ip_mse|. */
enum { TQO_SYM_LIGHT = 0, TQO_SYM_FULL = 1, TQO_SYM_FULL_PREPARED = 2 };
void tqo_distance_m_to_n_symmetric_qjl(const tqo_space *sp, const uint8_t *A, size_t m,
                                       const uint8_t *B, size_t n, float *out, int variant,
                                       int num_threads);
/* prepareSymmetricQuery: recon_q, sign_q (padded_dim each) and
 * s = {norm, gamma, sigma, scale * gamma, (pi / (2 D)) * gamma}. */
void tqo_prepare_symmetric(const tqo_space *sp, const uint8_t *code, float *recon_q,
                           float *sign_q, float *s);
/* distanceBatch1ToNSymmetricFull (:544-553) on a prepared row code. */
void tqo_distance_1_to_n_symmetric_full(const tqo_space *sp, const float *recon_q,
                                        const float *sign_q, const float *s,
                                        const uint8_t *B, size_t n, float *out,
                                        int num_threads);
double tqo_distance_symmetric_qjl_f64(const tqo_space *sp, const uint8_t *a, const uint8_t *b,
                                      int variant);

#ifdef __cplusplus
}
#endif
#endif /* TQ_ORACLE_H */
