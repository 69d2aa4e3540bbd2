// ref_shim.cpp -- a C entry point onto the reference library itself.
//
// TEST INFRASTRUCTURE ONLY.  Compiled (oracle/Makefile, target `ref`) together
// with the reference's own header-only sources, read in place, with the
// reference's pinned Release flags, into oracle/_ref/libtqref.so.  It exposes
// the reference's TurboQuantSpace (include/turboquant/space_turbo_quant.h:207)
// and its free helpers through plain C symbols so that the restatement in
// tq_oracle.c can be pinned against it with ctypes.
#include "turboquant/space_turbo_quant.h"

#include <cstring>

using turboquant::TurboQuantSpace;

extern "C" {

__attribute__((visibility("default"))) void *tqr_create(size_t dim, int bits, uint64_t rot_seed,
                                                         uint64_t qjl_seed, int num_threads) {
    return new TurboQuantSpace(dim, bits, rot_seed, qjl_seed, num_threads);
}

__attribute__((visibility("default"))) void tqr_destroy(void *sp) {
    delete static_cast<TurboQuantSpace *>(sp);
}

__attribute__((visibility("default"))) size_t tqr_code_size(const void *sp) {
    return static_cast<const TurboQuantSpace *>(sp)->codeSizeBytes();
}

__attribute__((visibility("default"))) size_t tqr_padded_dim(const void *sp) {
    return static_cast<const TurboQuantSpace *>(sp)->paddedDim();
}

__attribute__((visibility("default"))) float tqr_scale(const void *sp) {
    return static_cast<const TurboQuantSpace *>(sp)->scale();
}

// centroids: 2^(bits-1) floats; boundaries: 2^(bits-1)-1 floats;
// rot_signs / qjl_signs: padded_dim floats each.
__attribute__((visibility("default"))) void tqr_tables(const void *spv, float *centroids,
                                                        float *boundaries, float *rot_signs,
                                                        float *qjl_signs) {
    const auto *sp = static_cast<const TurboQuantSpace *>(spv);
    const int L = sp->numLevels();
    std::memcpy(centroids, sp->centroids(), sizeof(float) * L);
    auto table = turboquant::computeLloydMax(sp->bitsPerCoord() - 1);
    std::memcpy(boundaries, table.boundaries.data(), sizeof(float) * table.boundaries.size());
    auto rs = turboquant::generateSigns(sp->paddedDim(), sp->rotSeed());
    std::memcpy(rot_signs, rs.data(), sizeof(float) * rs.size());
    std::memcpy(qjl_signs, sp->qjlSigns(), sizeof(float) * sp->paddedDim());
}

__attribute__((visibility("default"))) void tqr_encode_batch(const void *sp, const float *X,
                                                              size_t n, uint8_t *out) {
    static_cast<const TurboQuantSpace *>(sp)->encodeBatch(X, n, out);
}

// norms[0] = |q|^2, norms[1] = |q|
__attribute__((visibility("default"))) void tqr_prepare_query(const void *sp, const float *q,
                                                               float *q_rot, float *s_q,
                                                               float *norms) {
    auto pq = static_cast<const TurboQuantSpace *>(sp)->prepareQuery(q);
    std::memcpy(q_rot, pq.q_rot.data(), sizeof(float) * pq.q_rot.size());
    std::memcpy(s_q, pq.s_q.data(), sizeof(float) * pq.s_q.size());
    norms[0] = pq.q_norm_sq;
    norms[1] = pq.q_norm;
}

__attribute__((visibility("default"))) void tqr_distance_1_to_n(const void *sp, const float *q,
                                                                 const uint8_t *codes, size_t n,
                                                                 float *out) {
    static_cast<const TurboQuantSpace *>(sp)->distanceBatch1ToN(q, codes, n, out);
}

__attribute__((visibility("default"))) void tqr_distance_m_to_n(const void *sp, const float *Q,
                                                                 size_t m, const uint8_t *codes,
                                                                 size_t n, float *out) {
    static_cast<const TurboQuantSpace *>(sp)->distanceBatchMToN(Q, m, codes, n, out);
}

__attribute__((visibility("default"))) void tqr_distance_m_to_n_symmetric(
    const void *sp, const uint8_t *A, size_t m, const uint8_t *B, size_t n, float *out) {
    static_cast<const TurboQuantSpace *>(sp)->distanceBatchMToNSymmetric(A, m, B, n, out);
}

}  // extern "C"
