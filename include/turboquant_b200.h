/*
 * turboquant_b200.h -- C ABI of the B200 (sm_100a) TurboQuant encode-and-scan
 * library, libtqb200.so.
 *
 * This is the drop-in boundary for the reference's TurboQuantSpace
 * (include/turboquant/space_turbo_quant.h:207-648) as its Python binding uses
 * it (python/turboquant/bindings.cpp:53-218).  The reference exposes no C ABI
 * (it is header-only C++ bound straight into pybind11); each function below
 * names the reference member and binding it replaces.  Plain pointers and
 * sizes only: no C++ or torch types cross this boundary, no exception escapes
 * it, and every function reports failure through a tq_status plus a
 * thread-local message (tq_last_error()).
 *
 * Codes are byte-identical to the reference layout: for padded dimension D
 * (the next power of two >= max(dim, 4)) a code is `packed_bytes` of units
 * unit = (sq_idx << 1) | qjl_bit -- two units per byte, even coordinate in the
 * low nibble, when bits_per_coord <= 4; one unit per byte otherwise -- followed
 * by the FP32 trailer [norm, gamma, sigma] (turbo_quant.h:101-185).
 *
 * Two families of entry points:
 *   - host-pointer functions (tq_encode_batch, tq_distance_*) behave like the
 *     reference methods: synchronous, all buffers in host memory, owned by the
 *     caller.  Large inputs are streamed through the GPU in chunks.
 *   - *_device functions take device pointers and a cudaStream_t (passed as
 *     void*; NULL = the legacy default stream) and are stream-ordered: they
 *     return once the work is enqueued.
 */
#ifndef TURBOQUANT_B200_H
#define TURBOQUANT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tq_status {
    TQ_OK = 0,
    TQ_ERR_INVALID_ARGUMENT = 1, /* bad size/shape/value; the Python mirror raises ValueError */
    TQ_ERR_CUDA = 2,             /* a CUDA runtime error (text in tq_last_error()) */
    TQ_ERR_OUT_OF_MEMORY = 3,    /* device or pinned-host allocation failed */
    TQ_ERR_NO_DEVICE = 4,        /* no usable sm_100 device */
    TQ_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up */
    TQ_ERR_BUSY = 6,             /* serving: a request was refused by admission */
    TQ_ERR_NOT_SUPPORTED = 7     /* valid request this build does not implement */
} tq_status;

/* Arithmetic used by the M x N contractions. */
typedef enum tq_precision {
    TQ_PRECISION_FP32 = 0,       /* FP32 CUDA-core kernels: the drop-in */
    TQ_PRECISION_SPLIT_BF16 = 1, /* tcgen05 tensor cores on hi+lo BF16 pairs, FP32 TMEM accumulators */
    TQ_PRECISION_SPLIT_TF32 = 2, /* tcgen05 tensor cores on hi+lo TF32 pairs, FP32 TMEM accumulators
                                    (the QJL-corrected symmetric distances only) */
    TQ_PRECISION_REFERENCE = 3,  /* the reference's own FP32 arithmetic in its Release build's
                                    summation order, one pair per thread: bit-identical to
                                    distSearchScalarB4 / distSearchAVX (asymmetric M x N) and
                                    distBuildScalarB4 / distBuildAVX (symmetric M x N) */
    TQ_PRECISION_SPLIT_BF16_DECODED = 4 /* as SPLIT_BF16, but the column tiles are decoded from
                                    the codes in shared memory (128 x 128 tiles) instead of
                                    being read from BF16 planes written to device memory
                                    first: 16 bytes of per-code scalars instead of 3-6 KB of
                                    planes per code.  Padded dims >= 64; a tile of 128 codes
                                    must fit in shared memory beside the pipeline (nibble
                                    codes up to padded dim 1024, byte codes up to 512);
                                    device codes 16-byte aligned.  Otherwise
                                    TQ_ERR_NOT_SUPPORTED.  Plain M x N entry points only. */
} tq_precision;

/* The QJL-corrected symmetric distances (space_turbo_quant.h:483-572, 731-945). */
typedef enum tq_sym_variant {
    TQ_SYM_LIGHT = 0,        /* distBuildLightScalar (:902-945): MSE + sign-agreement term */
    TQ_SYM_FULL = 1,         /* distBuildFullScalar (:731-800): all four inner-product terms */
    TQ_SYM_FULL_PREPARED = 2 /* distBuildFullPreparedScalar (:808-878): row code prepared once */
} tq_sym_variant;

typedef struct tq_space tq_space;

typedef struct tq_space_info {
    size_t dim;          /* TurboQuantSpace::dim()            space_turbo_quant.h:315 */
    size_t padded_dim;   /* TurboQuantSpace::paddedDim()      :316 */
    size_t packed_bytes; /* TurboQuantSpace::packedBytes()    :320 */
    size_t code_size;    /* TurboQuantSpace::codeSizeBytes()  :319 */
    int bits_per_coord;  /* TurboQuantSpace::bitsPerCoord()   :321 */
    int num_levels;      /* TurboQuantSpace::numLevels()      :323 */
    int padded;          /* TurboQuantSpace::padded()         :317 */
    int num_threads;     /* TurboQuantSpace::numThreads()     :318 (host threads; kept for API parity) */
    int device;          /* CUDA device the space's tables live on */
    uint64_t rot_seed;   /* :326 */
    uint64_t qjl_seed;   /* :327 */
    float scale;         /* TurboQuantSpace::scale()          :324 */
} tq_space_info;

/* Message of the last failing call on this thread ("" if none). */
const char *tq_last_error(void);
const char *tq_version(void);

/* Replaces TurboQuantSpace::TurboQuantSpace (space_turbo_quant.h:250-311),
 * bound at bindings.cpp:60-65.  Builds the Lloyd-Max table and both sign
 * vectors on the host and uploads them to `device` (-1 = current device).
 * Unlike the reference (asserts compiled out), dim < 1 or bits outside 2..9
 * return TQ_ERR_INVALID_ARGUMENT.  The padding warning of :269-273 is printed
 * to stderr the same way. */
tq_status tq_space_create(size_t dim, int bits_per_coord, uint64_t rot_seed,
                          uint64_t qjl_seed, int num_threads, int device,
                          tq_space **out);
void tq_space_destroy(tq_space *sp);
tq_status tq_space_get_info(const tq_space *sp, tq_space_info *info);

/* Host copies of the tables: centroids[num_levels], boundaries[num_levels-1],
 * rot_signs[padded_dim], qjl_signs[padded_dim] (any pointer may be NULL).
 * computeLloydMax space_turbo_quant.h:76-131; generateSigns turbo_quant.h:74-86. */
tq_status tq_space_tables(const tq_space *sp, float *centroids, float *boundaries,
                          float *rot_signs, float *qjl_signs);

/* quantize (space_turbo_quant.h:332-337) of n normalised values on the host,
 * through the same bucket table the encode kernel uses for bits >= 6 (the
 * direct count otherwise).  A diagnostic: it lets the table's exactness be
 * checked without a GPU.  idx[i] = #{j : z[i] > boundaries[j]} as uint8. */
tq_status tq_space_quantize(const tq_space *sp, const float *z, size_t n, uint8_t *idx);

/* ---- host-pointer entry points (synchronous) ----------------------------- */

/* TurboQuantSpace::encodeBatch (space_turbo_quant.h:400-407); bindings.cpp:93-116.
 * X: n x dim float32 row-major; out: n x code_size bytes.  Bit-exact. */
tq_status tq_encode_batch(const tq_space *sp, const float *X, size_t n, uint8_t *out);

/* TurboQuantSpace::distanceBatch1ToN (:577-585); bindings.cpp:156-172.
 * query: dim floats; codes: n codes; out: n floats. */
tq_status tq_distance_1_to_n(const tq_space *sp, const float *query, const uint8_t *codes,
                             size_t n, float *out);

/* TurboQuantSpace::distanceBatchMToN (:588-599); bindings.cpp:175-194.
 * queries: m x dim; out: m x n row-major. */
tq_status tq_distance_m_to_n(const tq_space *sp, const float *queries, size_t m,
                             const uint8_t *codes, size_t n, float *out,
                             tq_precision precision);

/* TurboQuantSpace::distanceBatchMToNSymmetric (:602-615); bindings.cpp:197-218.
 * MSE-only: gamma and the QJL bits are ignored, as in the reference. */
tq_status tq_distance_m_to_n_symmetric(const tq_space *sp, const uint8_t *codes_a, size_t m,
                                       const uint8_t *codes_b, size_t n, float *out,
                                       tq_precision precision);

/* ---- device-pointer entry points (stream-ordered) ------------------------ */

/* encodeBatch on device buffers. */
tq_status tq_encode_batch_device(const tq_space *sp, const float *X, size_t n, uint8_t *out,
                                 void *stream);

/* TurboQuantSpace::prepareQuery (:439-460) for m queries: q_rot and s_q are
 * m x padded_dim, norms is m x 2 = (|q|^2, |q|). */
tq_status tq_prepare_queries_device(const tq_space *sp, const float *queries, size_t m,
                                    float *q_rot, float *s_q, float *norms, void *stream);
/* TurboQuantSpace::prepareQuery (:439-460; bindings.cpp:268-273) of one query
 * on host pointers, synchronous: q_rot[padded_dim], s_q[padded_dim],
 * norms[2] = (|q|^2, |q|), bit-identical to the reference. */
tq_status tq_prepare_query(const tq_space *sp, const float *query, float *q_rot, float *s_q,
                           float *norms);

/* distanceBatch1ToN on device buffers.  Scratch for the prepared query is
 * taken from the stream-ordered pool of the device (cudaMallocAsync). */
tq_status tq_distance_1_to_n_device(const tq_space *sp, const float *query,
                                    const uint8_t *codes, size_t n, float *out, void *stream);

/* The scan alone, for a query already prepared by tq_prepare_queries_device
 * (q_rot, s_q: padded_dim floats; norms: 2 floats) -- the reference's
 * distance(const TurboQuantPreparedQuery&, code) (:465-468) over n codes.
 * Allocates nothing. */
tq_status tq_distance_1_to_n_prepared_device(const tq_space *sp, const float *q_rot,
                                             const float *s_q, const float *norms,
                                             const uint8_t *codes, size_t n, float *out,
                                             void *stream);

/* distance_1_to_n on device buffers for callers that cannot allocate device
 * memory: for example code that runs inside a memory budget fixed up front
 * (a serving process that reserved its pool at start-up), a framework
 * plug-in whose enqueue step is not allowed to allocate, or a latency path
 * that cannot afford the synchronisation of cudaMalloc/cudaFree.  It has no
 * counterpart in the reference (whose CPU code never allocates device memory).
 *
 * It computes exactly what tq_distance_1_to_n_device computes, but keeps the
 * prepared query (2 * padded_dim + 2 floats) in a fixed array that the
 * library holds in device memory on every GPU that loads it, until the
 * process exits: 16,386 floats (64 KiB + 8 bytes), enough for the largest
 * padded_dim this library supports (8192).  Larger requests are rejected
 * with TQ_ERR_INVALID_ARGUMENT.  No call allocates or frees device memory.
 *
 * The first call on a device looks up that device's copy of the array
 * (cudaGetSymbolAddress) and keeps its address for the life of the process;
 * make that first call before any stream capture.  A device reset
 * (cudaDeviceReset) may move the array, so this entry point must not be
 * called on a device after that device was reset.
 * All calls on a device share the one array, and it keeps the last call's
 * contents; each call rewrites every value it reads before reading it, so
 * nothing needs clearing.  Calls whose work overlaps on the GPU (different
 * streams, or different host threads without ordering) race on the array:
 * order them on one stream or serialise them. */
tq_status tq_distance_1_to_n_device_noalloc(const tq_space *sp, const float *query,
                                            const uint8_t *codes, size_t n, float *out,
                                            void *stream);

/* distanceBatchMToN on device buffers. */
tq_status tq_distance_m_to_n_device(const tq_space *sp, const float *queries, size_t m,
                                    const uint8_t *codes, size_t n, float *out,
                                    tq_precision precision, void *stream);

/* distanceBatchMToNSymmetric on device buffers. */
tq_status tq_distance_m_to_n_symmetric_device(const tq_space *sp, const uint8_t *codes_a,
                                              size_t m, const uint8_t *codes_b, size_t n,
                                              float *out, tq_precision precision,
                                              void *stream);

/* ---- beside the encode-and-scan path ------------------------------------ */

/* rotatedCoordsBatch (space_turbo_quant.h:411-435; bindings.cpp:119-132):
 * out[n, padded_dim] = the sigma-normalised post-rotation coordinates,
 * bit-identical to the reference.  Host pointers, synchronous. */
tq_status tq_rotated_coords_batch(const tq_space *sp, const float *X, size_t n, float *out);
/* The same on device buffers, stream-ordered. */
tq_status tq_rotated_coords_batch_device(const tq_space *sp, const float *X, size_t n, float *out,
                                         void *stream);

/* distanceBatchMToNSymmetric{Light,Full,FullPrepared} (:557-572, 618-647,
 * bindings.cpp:221-266, 312-334): out[m, n] row-major.  Host pointers,
 * synchronous.  Each code is reconstructed and passed through the QJL
 * Hadamard once; the pair terms are two contractions on the GPU:
 * TQ_PRECISION_FP32 on CUDA cores (the drop-in), TQ_PRECISION_SPLIT_TF32 on
 * tcgen05 tensor cores (hi/lo TF32 operands, FP32 accumulators; padded dims
 * below 64 stay on CUDA cores).  TQ_PRECISION_SPLIT_BF16 is refused with
 * TQ_ERR_NOT_SUPPORTED: the operands are values of the small centroid table,
 * whose BF16-pair rounding errors add up instead of averaging out. */
tq_status tq_distance_m_to_n_symmetric_qjl(const tq_space *sp, const uint8_t *codes_a, size_t m,
                                           const uint8_t *codes_b, size_t n, float *out,
                                           tq_sym_variant variant, tq_precision precision);
/* The same on device buffers, stream-ordered. */
tq_status tq_distance_m_to_n_symmetric_qjl_device(const tq_space *sp, const uint8_t *codes_a,
                                                  size_t m, const uint8_t *codes_b, size_t n,
                                                  float *out, tq_sym_variant variant,
                                                  tq_precision precision, void *stream);

/* prepareSymmetricQuery (:499-535; bindings.cpp:276-282) of one code (host
 * pointers): recon_q[padded_dim] = RHT_qjl(c * sigma), sign_q[padded_dim] =
 * +-1, scalars[5] = {norm, gamma, sigma, scale * gamma, (pi / 2D) * gamma}. */
tq_status tq_prepare_symmetric_query(const tq_space *sp, const uint8_t *code, float *recon_q,
                                     float *sign_q, float *scalars);
/* distanceBatch1ToNSymmetricFull (:544-553; bindings.cpp:293-310) on a
 * prepared code.  Host pointers, synchronous. */
tq_status tq_distance_1_to_n_symmetric_full(const tq_space *sp, const float *recon_q,
                                            const float *sign_q, const float *scalars,
                                            const uint8_t *codes, size_t n, float *out);
/* The same with every buffer in device memory, stream-ordered. */
tq_status tq_distance_1_to_n_symmetric_full_device(const tq_space *sp, const float *recon_q,
                                                   const float *sign_q, const float *scalars,
                                                   const uint8_t *codes, size_t n, float *out,
                                                   void *stream);

/* The device status word of the space's stream-ordered kernels.  Every wait in
 * the staged 1->N scan is bounded; a wait that gives up (a copy that never
 * completes) writes a non-zero code here and the kernel returns without
 * finishing its codes.  Synchronise the streams the space's *_device calls ran
 * on, then call this: it reports the code in *code (0 = none), clears it, and
 * returns TQ_ERR_TIMEOUT when it was set.  The host-pointer entry points check
 * it themselves.  No counterpart in the reference (CPU code never waits on a
 * device). */
tq_status tq_space_take_device_status(const tq_space *sp, int *code);

/* Kernel timer of the 1->N scan (no counterpart in the reference: a
 * measurement aid).  While enabled, tq_distance_1_to_n_device and
 * tq_distance_1_to_n_prepared_device record a pair of CUDA events around
 * their scan kernel on the call's stream; enabling resets the record.
 * tq_space_scan_timer_read waits for the recorded launches and returns their
 * summed kernel time in milliseconds and their count. */
tq_status tq_space_scan_timer(tq_space *sp, int enable);
tq_status tq_space_scan_timer_read(tq_space *sp, double *total_ms, uint64_t *launches);

/* Self-test of the device-side failure path: a kernel waits, with a limit of
 * about budget_ms, on a barrier that nothing signals.  Returns TQ_ERR_TIMEOUT
 * when the wait gave up and reported it (the expected outcome; the context
 * stays usable), TQ_OK if it did not. */
tq_status tq_selftest_bounded_wait(int device, int budget_ms);

/* ---- serving: device-resident index + continuous-batching top-k server ---
 * The reference has no index or serving loop (README.md:81-83); these entry
 * points serve exact top-k asymmetric search over a corpus kept in HBM.  The
 * results are the stable argsort of the reference's own distances
 * (distSearchScalarB4 / distSearchAVX, space_turbo_quant.h:951-983 and
 * :1457-1539, in its Release build's summation order): ascending distance,
 * ties broken by the smaller code index, bit-identical distances, the same
 * whatever batch a request shares. */
typedef struct tq_index tq_index;
typedef struct tq_server tq_server;
typedef struct tq_request tq_request;

typedef struct tq_server_stats {
    uint64_t submitted, rejected, completed, batches, rows;
    size_t queued_rows;
    int slots, max_rows;
    int candidates;              /* tensor-pass candidates per query row */
    uint64_t fallback_rows;      /* rows the certificate left open, answered by an exact pass */
    uint64_t bound_violations;   /* candidates whose two distances differed by more than the bound */
    size_t pool_rows;            /* query rows of the admission pool (device memory) */
    size_t pool_used_rows;       /* rows held by queued and in-flight requests */
    uint64_t scan_pass_rows;     /* open rows answered by an exact scan of every code (the others
                                    by rescoring a tensor-core threshold pass's list) */
    uint64_t list_pass_rows;     /* of those, rows with more codes at or below their threshold
                                    than the scan collects, answered by a full list pass */
} tq_server_stats;

/* How an index keeps its corpus for the tensor-core pass. */
typedef enum tq_index_layout {
    TQ_INDEX_PLANES = 0, /* the codes plus their exact-sign hi/lo BF16 operand planes:
                            code_size + 6 * padded_dim + 8 bytes a code; the fastest pass */
    TQ_INDEX_CODES = 1   /* the codes plus four floats a code (code_size + 16 bytes): the pass
                            decodes each tile of codes in shared memory (kernel variants 1..4),
                            for corpora ~10x larger per GPU at a slower pass; padded dim >= 64 */
} tq_index_layout;

/* Keep n codes (host or device memory) resident in HBM in the given layout. */
tq_status tq_index_create_ex(const tq_space *sp, const uint8_t *codes, size_t n, int codes_on_device,
                             tq_index_layout layout, tq_index **out);
/* tq_index_create_ex with TQ_INDEX_PLANES. */
tq_status tq_index_create(const tq_space *sp, const uint8_t *codes, size_t n, int codes_on_device,
                          tq_index **out);
void tq_index_destroy(tq_index *ix);

typedef struct tq_server_params {
    int k;              /* results per query row, 1..16 */
    int max_rows;       /* query rows per batch, a positive multiple of 128 */
    int slots;          /* batches in flight, 1..8 (fewer if they do not fit in half of the
                           free device memory) */
    int kernel_variant; /* -1: autotune the contraction's tile shape per batch-size bucket;
                           else fixed (tq_topk_variant_shape): 0..6 for a TQ_INDEX_PLANES
                           index, 1..4 for TQ_INDEX_CODES */
    size_t queue_rows;  /* queued query rows beyond which submit returns TQ_ERR_BUSY
                           (0: no cap beyond the admission pool) */
    int candidates;     /* tensor-pass candidates per row that the exact stage rescores,
                           k..32 (0: min(32, k + 16)) */
    float bound_scale;  /* multiplier on the certificate's error bound (0: 1); a larger
                           value sends more rows to the exact full pass */
    size_t memory_budget; /* device bytes of the admission pool that holds the queries of
                           the queued and in-flight requests, dim * 4 bytes a row (0: an
                           eighth of the free device memory, at most 16 x max_rows rows);
                           submit returns TQ_ERR_BUSY when a request's rows do not fit */
} tq_server_params;

/* A server answering exact top-k for requests of up to max_rows queries:
 * a tcgen05 split-BF16 pass keeps `candidates` per row, a rescoring kernel
 * recomputes them with the reference's arithmetic and certifies the top-k
 * against the pass's error bound, and rows it cannot certify get an exact
 * full pass over the codes. */
tq_status tq_server_create_ex(tq_index *ix, const tq_server_params *params, tq_server **out);
/* tq_server_create_ex with candidates = 0 and bound_scale = 0. */
tq_status tq_server_create(tq_index *ix, int k, int max_rows, int slots, int kernel_variant,
                           size_t queue_rows, tq_server **out);
/* Queue m query rows (m x dim float32, copied); non-blocking. */
tq_status tq_server_submit(tq_server *sv, const float *queries, size_t m, tq_request **out);
/* Wait (timeout_ms < 0: forever) and copy the m x k results and the latency. */
tq_status tq_request_wait(tq_request *r, int timeout_ms, float *dist, int64_t *idx,
                          double *latency_ms);
int tq_request_done(tq_request *r);
void tq_request_release(tq_request *r);
/* Counters and up to `cap` recorded request latencies (milliseconds). */
tq_status tq_server_get_stats(tq_server *sv, tq_server_stats *out, float *latencies, size_t cap,
                          size_t *n_latencies);
tq_status tq_server_reset_stats(tq_server *sv);
/* The autotuner's choice per bucket: rows, kernel variant, and its measured ms
   per batch (two slots' launches overlapped, as the server runs them). */
tq_status tq_server_tuning(tq_server *sv, int *bucket_rows, int *variant, float *ms, int cap,
                           int *n);
/* Every time the autotuner took, bucket-major: ms[b * n_variants + v]
   (0 where a variant was not timed); from_cache = 1 when this server reused
   the process's earlier tuning of the same index shape, candidates and
   bucket rows. */
tq_status tq_server_tuning_times(tq_server *sv, float *ms, int cap, int *n_buckets, int *n_variants,
                                 int *from_cache);
/* The tile shape of a kernel variant: shape[0] query rows per CTA, shape[1]
   codes per tile (per pipeline stage), shape[2] pipeline stages, shape[3] K
   blocks of 64 per promoted accumulation chunk (0: the whole K in one
   accumulator, whose wider error bound the exact stage's certificate uses). */
tq_status tq_topk_variant_shape(int variant, int *shape);
void tq_server_destroy(tq_server *sv);

#ifdef __cplusplus
}
#endif
#endif /* TURBOQUANT_B200_H */
