// tq_serve.cu -- device-resident index and the continuous-batching search server.
//
// The reference has no index or serving loop (README.md:81-83); this is the
// north-star serving path built on the same distance contraction:
//
//   tq_index   the corpus itself resident in HBM (the exact stages read it)
//              and, by layout:
//              TQ_INDEX_PLANES: the codes decoded once into exact-sign hi/lo
//                BF16 planes B[j] = [sigma_j c[idx_j] / g_j | (+-1)_j] (K = 2D;
//                6 D + 8 more bytes a code) with c1 = g |x| and c2 = |x|^2;
//              TQ_INDEX_CODES: four floats a code (c1, c2 and the chunk
//                factors fc, fs of launch_dec_factors); the tensor pass decodes
//                each B tile in shared memory from the codes.
//   slot       buffers for one batch of up to `max_rows` query rows and one CUDA
//              graph per row bucket (128, 256, 512, ... max_rows) capturing
//              rows gathered from the pool -> prepareQuery -> query planes ->
//              tcgen05 candidates (B decoded in shared memory) ->
//              merge -> D2H results; the kernels read the batch's row count
//              from device memory, so the graph replays for any batch size.
//   server     a scheduler thread.  Requests are queued on submit; whenever a
//              slot is free the queued requests are packed in arrival order
//              into one batch (continuous batching: requests that arrive while
//              other batches are on the GPU join the next batch) and the
//              bucket's graph is launched on the slot's stream.  Slots run on
//              separate streams, so one batch's copies and query preparation
//              overlap another's contraction.
//   admission  an admitted request's queries are copied at submit into a
//              device pool of query rows whose size is the server's memory
//              budget (by default a share of the device's free memory at
//              creation); submit refuses a request (TQ_ERR_BUSY) when its rows
//              do not fit in the pool's free space, which holds the rows of the
//              queued and the in-flight requests.  A batch gathers its rows
//              from the pool on the device.
//   autotune   per bucket, each kernel variant (tile shape x stage depth) is
//              timed on the index and the fastest is captured into the graph.
//   exact      the tensor-core pass keeps `kc` candidates per row; the
//              rescoring kernel recomputes them with the reference's own
//              arithmetic (tq_exact.cu) and certifies the row's top-k with the
//              pass's error bound; rows it cannot certify are answered by an
//              exact full pass over the codes.  Results are therefore the
//              stable argsort of the reference's distances, whatever the
//              batch they ran in.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdint>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "tq_exact.h"
#include "tq_host.h"
#include "tq_mton.h"

struct tq_index {
    tq_space *sp = nullptr;
    size_t n = 0, n_pad = 0;
    int K = 0;
    int layout = TQ_INDEX_PLANES;
    int K_lo = 0;             // PLANES: columns of the lo plane (tq::asym_lo_width)
    void *block = nullptr;    // one allocation: [planes], c1, c2, [fc, fs], codes, bound
    void *planes = nullptr;   // PLANES: hi plane n_pad x K, then lo plane n_pad x K_lo, BF16
    float *c1 = nullptr, *c2 = nullptr, *fc = nullptr, *fs = nullptr;
    uint8_t *codes = nullptr;  // the corpus itself (n x code_size), for the exact stages
    float *bound = nullptr;    // kBoundFloats index-wide maxima of the error bound
    float cmax = 0.0f;         // max |centroid|
    int device = -1;
};

namespace {

using tq::cuda_fail;
using tq::DeviceGuard;
using tq::fail;

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct tq_request {
    std::vector<float> queries;  // m x dim
    size_t m = 0;
    size_t pool_off = 0;                // first row of its queries in the server's pool
    cudaEvent_t uploaded = nullptr;     // the copy into the pool is done
    int k = 0;
    std::vector<float> dist;     // m x k
    std::vector<long long> idx;  // m x k
    double t_submit = 0, t_done = 0;
    tq_status status = TQ_OK;
    bool done = false;
    std::mutex mu;
    std::condition_variable cv;
};

namespace {

struct Slot {
    int max_rows = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    float *h_q = nullptr;
    int *h_m = nullptr;
    int *h_err = nullptr;
    float *h_d = nullptr;
    long long *h_i = nullptr;
    void *d_block = nullptr;  // one device allocation for all buffers below
    float *d_q = nullptr, *d_prep = nullptr, *d_r1 = nullptr, *d_r2 = nullptr, *d_pd = nullptr,
          *d_od = nullptr, *d_cd = nullptr, *d_fpd = nullptr, *d_thr = nullptr, *d_colld = nullptr,
          *d_tthr = nullptr, *d_r1o = nullptr, *d_r2o = nullptr;
    int *d_m = nullptr, *d_pi = nullptr, *d_err = nullptr, *d_fail = nullptr, *d_cnt = nullptr,
        *d_fpi = nullptr, *d_colln = nullptr, *d_colli = nullptr, *d_scan = nullptr,
        *d_list_rows = nullptr;
    void *d_ap2 = nullptr;  // the open rows' query planes (same shape as d_ap)
    unsigned long long *d_gthr = nullptr;  // per row: the top-k pass's published bound
    long long *d_ci = nullptr;
    int *h_cnt = nullptr;  // pinned copy of d_cnt after each batch
    int *h_rows = nullptr;  // pool row of each batch row (pinned)
    int *d_rows = nullptr;
    void *d_ap = nullptr;  // query planes: max_rows x K x 2 BF16 planes
    long long *d_oi = nullptr;
    std::vector<int> bucket_rows;
    std::vector<cudaGraphExec_t> graphs;
    std::vector<tq_request *> batch;  // requests in flight in this slot
    size_t batch_rows = 0;
    bool busy = false;
};

}  // namespace

struct tq_server {
    tq_index *index = nullptr;
    int k = 10;
    int kc = 26;              // tensor-pass candidates per row
    float bound_scale = 1.0f; // multiplier on the certificate's error bound
    int fb_ctas = 296;        // CTAs of the exact fallback pass
    int grid = 148;
    int max_rows = 1024;
    size_t queue_rows_cap = 0;
    std::vector<Slot> slots;
    std::vector<int> bucket_variant;  // autotuned kernel variant per bucket
    std::vector<double> bucket_ms;
    std::vector<float> tune_ms;       // bucket x variant times (0: not timed)
    bool tuned_from_cache = false;
    std::deque<tq_request *> pending;
    size_t pending_rows = 0;
    // admission pool: pool_rows query rows in device memory, first-fit ranges
    float *pool = nullptr;
    size_t pool_rows = 0, pool_used = 0;
    std::map<size_t, size_t> pool_free;  // offset -> length
    cudaStream_t up_stream = nullptr;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    // stats
    uint64_t submitted = 0, rejected = 0, completed = 0, batches = 0, rows_done = 0;
    uint64_t fallback_rows = 0, bound_violations = 0, scan_pass_rows = 0, list_pass_rows = 0;
    std::vector<float> latencies_ms;  // ring of the most recent completions
    size_t lat_pos = 0;
    double busy_ms = 0;
};

namespace {

// Kernel variants that serve an index layout: any for planes, the decoded-B
// ones for codes.
bool variant_fits(const tq_index *ix, int v) {
    return ix->layout == TQ_INDEX_CODES ? tq::tc_topk_dec_ok(v, (int)ix->sp->code_size)
                                        : (v >= 0 && v < tq::tc_topk_variants());
}

int bucket_index(const tq_server *sv, size_t rows) {
    const auto &b = sv->slots[0].bucket_rows;
    for (size_t i = 0; i < b.size(); ++i)
        if (rows <= (size_t)b[i]) return (int)i;
    return (int)b.size() - 1;
}

// First-fit allocation of `m` pool rows (caller holds sv->mu).
bool pool_alloc(tq_server *sv, size_t m, size_t *off) {
    for (auto it = sv->pool_free.begin(); it != sv->pool_free.end(); ++it) {
        if (it->second < m) continue;
        *off = it->first;
        const size_t rest = it->second - m;
        const size_t at = it->first + m;
        sv->pool_free.erase(it);
        if (rest) sv->pool_free.emplace(at, rest);
        sv->pool_used += m;
        return true;
    }
    return false;
}

// Returns rows [off, off + m) to the pool, merging with free neighbours
// (caller holds sv->mu).
void pool_release(tq_server *sv, size_t off, size_t m) {
    auto nx = sv->pool_free.lower_bound(off);
    if (nx != sv->pool_free.begin()) {
        auto pv = std::prev(nx);
        if (pv->first + pv->second == off) {
            off = pv->first;
            m += pv->second;
            sv->pool_free.erase(pv);
        }
    }
    if (nx != sv->pool_free.end() && off + m == nx->first) {
        m += nx->second;
        sv->pool_free.erase(nx);
    }
    sv->pool_free.emplace(off, m);
}

void release_request_rows(tq_server *sv, tq_request *r) {
    pool_release(sv, r->pool_off, r->m);
    sv->pool_used -= r->m;
    if (r->uploaded) cudaEventDestroy(r->uploaded);
    r->uploaded = nullptr;
}

// Enqueue the batch pipeline of `rows_cap` rows with kernel variant `var` on
// the slot's stream (used both for graph capture and for autotuning runs).
cudaError_t enqueue_batch(tq_server *sv, Slot &sl, int rows_cap, int var, bool copies) {
    tq_index *ix = sv->index;
    tq_space *sp = ix->sp;
    const size_t D = sp->D;
    const size_t K = (size_t)ix->K;
    cudaStream_t st = sl.stream;
    cudaError_t e = cudaSuccess;
    if (copies) {
        // the batch's rows: their pool rows, then a gather from the pool
        e = cudaMemcpyAsync(sl.d_rows, sl.h_rows, (size_t)rows_cap * sizeof(int), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.d_m, sl.h_m, sizeof(int), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = tq::launch_gather_rows(sv->pool, sl.d_rows, sl.d_m, sp->dim, rows_cap, sl.d_q, st);
        if (e != cudaSuccess) return e;
    }
    float *q_rot = sl.d_prep, *s_q = q_rot + (size_t)rows_cap * D, *norms = s_q + (size_t)rows_cap * D;
    e = tq::launch_prepare(sp->P, sp->T, sl.d_q, rows_cap, q_rot, s_q, norms, st);
    if (e != cudaSuccess) return e;
    unsigned char *ah = static_cast<unsigned char *>(sl.d_ap);
    unsigned char *al = ah + (size_t)rows_cap * K * 2;
    e = tq::launch_planes_from_prepared(q_rot, s_q, norms, rows_cap, rows_cap, (int)D, tq::kPlaneBF16,
                                        ah, al, sl.d_r1, sl.d_r2, st);
    if (e != cudaSuccess) return e;
    // tensor-core pass: each row's kc best candidates by approximate distance
    const bool planes = ix->layout == TQ_INDEX_PLANES;
    unsigned char *bh = planes ? static_cast<unsigned char *>(ix->planes) : nullptr;
    unsigned char *bl = planes ? bh + ix->n_pad * K * 2 : nullptr;
    tq::DecSrc dec;  // codes layout: the column tiles decoded in shared memory
    if (!planes) {
        dec.codes = ix->codes;
        dec.n = (unsigned)ix->n;
        dec.cs = (int)sp->code_size;
        dec.nibble = sp->P.nibble;
        dec.kbc = (int)(D / 64);
        dec.fc = ix->fc;
        dec.fs = ix->fs;
        dec.centroids = sp->T.centroids;
        dec.levels = sp->levels;
    }
    e = cudaMemsetAsync(sl.d_gthr, 0xFF, (size_t)rows_cap * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (planes)
        e = tq::launch_tc_topk(var, ah, al, rows_cap, bh, bl, ix->n_pad, (int)K, ix->K_lo, sl.d_m, ix->n,
                               sl.d_r1, sl.d_r2, ix->c1, ix->c2, sv->kc, sl.d_pd, sl.d_pi, sl.d_gthr,
                               sl.d_err, sv->grid, st);
    else
        e = tq::launch_tc_topk_dec(var, ah, al, rows_cap, dec, ix->n_pad, (int)K, sl.d_m, ix->n,
                                   sl.d_r1, sl.d_r2, ix->c1, ix->c2, sv->kc, sl.d_pd, sl.d_pi, sl.d_gthr,
                                   sl.d_err, sv->grid, st);
    if (e != cudaSuccess) return e;
    e = tq::launch_topk_merge(sl.d_m, sv->grid, tq::tc_topk_lists(var), sl.d_pd, sl.d_pi, sv->kc,
                              rows_cap, sl.d_cd, sl.d_ci, st);
    if (e != cudaSuccess) return e;
    // exact stages: rescoring + certificate, then the full pass for the rows
    // the certificate leaves open
    e = cudaMemsetAsync(sl.d_cnt, 0, tq::kCntWords * sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = tq::launch_rescore(sp->P, sp->T.centroids, ix->cmax, sl.d_m, sv->kc, sv->k, sl.d_cd, sl.d_ci,
                           q_rot, s_q, norms, ix->codes, ix->n, ix->bound,
                           tq::tc_topk_kappa(var, (int)K, ix->K_lo),
                           tq::tc_topk_kappa(tq::tc_thresh_variant(!planes, ix->n_pad), (int)K, ix->K_lo),
                           sv->bound_scale, sl.d_od,
                           sl.d_oi, sl.d_fail, sl.d_thr, sl.d_tthr, sl.d_cnt, rows_cap, st);
    if (e != cudaSuccess) return e;
    // the open rows' threshold pass on the tensor cores (when enough are open)
    e = cudaMemsetAsync(sl.d_colln, 0, (size_t)rows_cap * sizeof(int), st);
    if (e != cudaSuccess) return e;
    unsigned char *ah2 = static_cast<unsigned char *>(sl.d_ap2);
    unsigned char *al2 = ah2 + (size_t)rows_cap * K * 2;
    e = tq::launch_gather_open(sl.d_cnt, sl.d_fail, ah, al, sl.d_r1, sl.d_r2, (int)K, rows_cap, ah2, al2,
                               sl.d_r1o, sl.d_r2o, st);
    if (e != cudaSuccess) return e;
    e = tq::launch_tc_thresh(ah2, al2, rows_cap, bh, bl, planes ? nullptr : &dec, ix->n_pad, (int)K,
                             ix->K_lo, sl.d_cnt + tq::kCntFallbackRows, tq::kTensorTierMinRows, ix->n,
                             sl.d_r1o, sl.d_r2o, ix->c1, ix->c2, sl.d_tthr, sl.d_colln, sl.d_colli,
                             tq::kCollectCap, sl.d_err, sv->grid, st);
    if (e != cudaSuccess) return e;
    const tq::FallbackBuffers fb{sl.d_thr,  sl.d_tthr,      sl.d_colln, sl.d_colld, sl.d_colli,
                                 sl.d_scan, sl.d_list_rows, sl.d_fpd,   sl.d_fpi};
    e = tq::launch_fallback(sp->P, sp->T.centroids, sv->k, q_rot, s_q, norms, ix->codes, ix->n,
                            sl.d_fail, sl.d_cnt, sv->fb_ctas, true, fb, sl.d_od, sl.d_oi, rows_cap, st);
    if (e != cudaSuccess) return e;
    if (copies) {
        e = cudaMemcpyAsync(sl.h_d, sl.d_od, (size_t)rows_cap * sv->k * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.h_i, sl.d_oi, (size_t)rows_cap * sv->k * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_err, sl.d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.h_cnt, sl.d_cnt, tq::kCntWords * sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    return e;
}

tq_status slot_alloc(tq_server *sv, Slot &sl) {
    tq_index *ix = sv->index;
    tq_space *sp = ix->sp;
    const size_t R = (size_t)sv->max_rows, D = sp->D, K = (size_t)ix->K, k = (size_t)sv->k;
    sl.max_rows = sv->max_rows;
    TQ_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    TQ_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "cudaEventCreate");
    TQ_CUDA(cudaMallocHost(&sl.h_q, R * sp->dim * 4), "cudaMallocHost(queries)");
    TQ_CUDA(cudaMallocHost(&sl.h_m, 16), "cudaMallocHost(m)");
    TQ_CUDA(cudaMallocHost(&sl.h_err, 16), "cudaMallocHost(err)");
    *sl.h_err = 0;
    TQ_CUDA(cudaMallocHost(&sl.h_d, R * k * 4), "cudaMallocHost(dist)");
    TQ_CUDA(cudaMallocHost(&sl.h_i, R * k * 8), "cudaMallocHost(idx)");
    TQ_CUDA(cudaMallocHost(&sl.h_cnt, tq::kCntWords * sizeof(int)), "cudaMallocHost(counters)");
    TQ_CUDA(cudaMallocHost(&sl.h_rows, R * sizeof(int)), "cudaMallocHost(rows)");
    std::memset(sl.h_rows, 0, R * sizeof(int));
    std::memset(sl.h_cnt, 0, tq::kCntWords * sizeof(int));
    std::memset(sl.h_q, 0, R * sp->dim * 4);
    // device block layout (each part 256-byte aligned)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = round_up(off + bytes, 256);
        return o;
    };
    const size_t o_q = take(R * sp->dim * 4), o_m = take(16), o_prep = take(R * (2 * D + 2) * 4);
    const size_t o_ap = take(R * K * 4), o_r1 = take(R * 4), o_r2 = take(R * 4);
    const size_t parts = (size_t)sv->grid * 128 * tq::kTopKListsMax * tq::kCandMax;
    const size_t o_pd = take(parts * 4), o_pi = take(parts * 4), o_od = take(R * k * 4);
    const size_t o_oi = take(R * k * 8), o_err = take(16);
    const size_t kc = (size_t)sv->kc, fparts = R * (size_t)sv->fb_ctas * k;
    const size_t o_cd = take(R * kc * 4), o_ci = take(R * kc * 8), o_fail = take(R * 4);
    const size_t o_cnt = take(tq::kCntWords * 4), o_fpd = take(fparts * 4), o_fpi = take(fparts * 4);
    const size_t o_rows = take(R * 4), o_thr = take(R * 4), o_tthr = take(R * 4), o_colln = take(2 * R * 4);
    const size_t o_colld = take(R * tq::kCollectCap * 4), o_colli = take(R * tq::kCollectCap * 4);
    const size_t o_scan = take(R * 4), o_list = take(R * 4), o_ap2 = take(R * K * 4);
    const size_t o_r1o = take(R * 4), o_r2o = take(R * 4), o_gthr = take(R * 8);
    TQ_CUDA(cudaMalloc(&sl.d_block, off), "cudaMalloc(slot)");
    TQ_CUDA(cudaMemset(sl.d_block, 0, off), "cudaMemset(slot)");
    auto *base = static_cast<unsigned char *>(sl.d_block);
    sl.d_q = reinterpret_cast<float *>(base + o_q);
    sl.d_m = reinterpret_cast<int *>(base + o_m);
    sl.d_prep = reinterpret_cast<float *>(base + o_prep);
    sl.d_ap = base + o_ap;
    sl.d_r1 = reinterpret_cast<float *>(base + o_r1);
    sl.d_r2 = reinterpret_cast<float *>(base + o_r2);
    sl.d_pd = reinterpret_cast<float *>(base + o_pd);
    sl.d_pi = reinterpret_cast<int *>(base + o_pi);
    sl.d_od = reinterpret_cast<float *>(base + o_od);
    sl.d_oi = reinterpret_cast<long long *>(base + o_oi);
    sl.d_err = reinterpret_cast<int *>(base + o_err);
    sl.d_cd = reinterpret_cast<float *>(base + o_cd);
    sl.d_ci = reinterpret_cast<long long *>(base + o_ci);
    sl.d_fail = reinterpret_cast<int *>(base + o_fail);
    sl.d_cnt = reinterpret_cast<int *>(base + o_cnt);
    sl.d_fpd = reinterpret_cast<float *>(base + o_fpd);
    sl.d_fpi = reinterpret_cast<int *>(base + o_fpi);
    sl.d_rows = reinterpret_cast<int *>(base + o_rows);
    sl.d_thr = reinterpret_cast<float *>(base + o_thr);
    sl.d_tthr = reinterpret_cast<float *>(base + o_tthr);
    sl.d_colln = reinterpret_cast<int *>(base + o_colln);
    sl.d_colld = reinterpret_cast<float *>(base + o_colld);
    sl.d_colli = reinterpret_cast<int *>(base + o_colli);
    sl.d_scan = reinterpret_cast<int *>(base + o_scan);
    sl.d_list_rows = reinterpret_cast<int *>(base + o_list);
    sl.d_ap2 = base + o_ap2;
    sl.d_r1o = reinterpret_cast<float *>(base + o_r1o);
    sl.d_r2o = reinterpret_cast<float *>(base + o_r2o);
    sl.d_gthr = reinterpret_cast<unsigned long long *>(base + o_gthr);
    for (int b = 128; b < sv->max_rows; b *= 2) sl.bucket_rows.push_back(b);
    sl.bucket_rows.push_back(sv->max_rows);
    return TQ_OK;
}

void slot_free(Slot &sl) {
    for (auto g : sl.graphs)
        if (g) cudaGraphExecDestroy(g);
    sl.graphs.clear();
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.d_block) cudaFree(sl.d_block);
    if (sl.h_q) cudaFreeHost(sl.h_q);
    if (sl.h_m) cudaFreeHost(sl.h_m);
    if (sl.h_err) cudaFreeHost(sl.h_err);
    if (sl.h_d) cudaFreeHost(sl.h_d);
    if (sl.h_i) cudaFreeHost(sl.h_i);
    if (sl.h_cnt) cudaFreeHost(sl.h_cnt);
    if (sl.h_rows) cudaFreeHost(sl.h_rows);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    sl = Slot();
}

// Time each kernel variant for each bucket the way the server runs it and
// keep the fastest.  Each slot (at most two) runs the bucket twice, the slots'
// launches alternating on their own streams, and the score is the time from
// the first start to the last end per batch: with two slots one batch's
// tail overlaps the next batch's start, which favours tiles that a single
// isolated launch would not.  The queries are non-zero (uniform in [-1, 1), a
// fixed LCG stream): MMAs on zero operands draw less power, so a tensor-bound
// variant would otherwise be timed at a clock that real batches under the
// power cap do not get.
// Tuning results of this process, per (device, padded dim, bits, corpus size,
// candidates, slots tuned together, bucket rows): the fastest variant and its
// time.  A server whose key is present skips timing that bucket.
struct TuneKey {
    int device, D, bits, kc, ns, rows, layout;
    size_t n;
    bool operator<(const TuneKey &o) const {
        return std::tie(device, D, bits, kc, ns, rows, layout, n) <
               std::tie(o.device, o.D, o.bits, o.kc, o.ns, o.rows, o.layout, o.n);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, double>> g_tune_cache;

tq_status autotune(tq_server *sv, int fixed_variant) {
    const int ns = std::min<int>(2, (int)sv->slots.size());
    Slot &s0 = sv->slots[0];
    const int nb = (int)s0.bucket_rows.size();
    const int nv = tq::tc_topk_variants();
    sv->bucket_variant.assign(nb, fixed_variant >= 0 ? fixed_variant : 4);  // 4 fits both layouts
    sv->bucket_ms.assign(nb, 0.0);
    sv->tune_ms.assign((size_t)nb * nv, 0.0f);
    const tq_index *ix = sv->index;
    auto key_of = [&](int rows) {
        return TuneKey{ix->device, (int)ix->sp->D, ix->sp->bits, sv->kc, ns, rows, ix->layout, ix->n};
    };
    if (fixed_variant < 0) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        bool all = true;
        for (int b = 0; b < nb; ++b) {
            auto it = g_tune_cache.find(key_of(s0.bucket_rows[b]));
            if (it == g_tune_cache.end()) {
                all = false;
                break;
            }
            sv->bucket_variant[b] = it->second.first;
            sv->bucket_ms[b] = it->second.second;
        }
        if (all) {
            sv->tuned_from_cache = true;
            return TQ_OK;
        }
    }
    const size_t qn = (size_t)s0.max_rows * sv->index->sp->dim;
    uint32_t x = 0x9E3779B9u;
    for (size_t i = 0; i < qn; ++i) {
        x = x * 1664525u + 1013904223u;
        s0.h_q[i] = (float)((int)(x >> 8) - (1 << 23)) * (1.0f / (float)(1 << 23));
    }
    for (int si = 0; si < ns; ++si) {
        Slot &sl = sv->slots[si];
        TQ_CUDA(cudaMemcpyAsync(sl.d_q, s0.h_q, qn * sizeof(float), cudaMemcpyHostToDevice, sl.stream),
                "H2D tuning queries");
        TQ_CUDA(cudaStreamSynchronize(sl.stream), "sync");
    }
    cudaEvent_t e0, e1[2];
    TQ_CUDA(cudaEventCreate(&e0), "event");
    TQ_CUDA(cudaEventCreate(&e1[0]), "event");
    TQ_CUDA(cudaEventCreate(&e1[1]), "event");
    constexpr int kReps = 1;
    for (int b = 0; b < nb; ++b) {
        const int rows = s0.bucket_rows[b];
        for (int si = 0; si < ns; ++si) {
            Slot &sl = sv->slots[si];
            *sl.h_m = rows;
            TQ_CUDA(cudaMemcpyAsync(sl.d_m, sl.h_m, sizeof(int), cudaMemcpyHostToDevice, sl.stream), "H2D m");
            TQ_CUDA(cudaStreamSynchronize(sl.stream), "sync");
        }
        double best = 1e30;
        for (int v = 0; v < nv; ++v) {
            if (fixed_variant >= 0 && v != fixed_variant) continue;
            if (!variant_fits(sv->index, v)) continue;
            TQ_CUDA(enqueue_batch(sv, s0, rows, v, false), "autotune warm-up");
            TQ_CUDA(cudaEventRecord(e0, s0.stream), "event");
            for (int si = 1; si < ns; ++si)
                TQ_CUDA(cudaStreamWaitEvent(sv->slots[si].stream, e0, 0), "stream wait");
            for (int r = 0; r < kReps; ++r)
                for (int si = 0; si < ns; ++si)
                    TQ_CUDA(enqueue_batch(sv, sv->slots[si], rows, v, false), "autotune run");
            float ms = 0;
            for (int si = 0; si < ns; ++si) {
                TQ_CUDA(cudaEventRecord(e1[si], sv->slots[si].stream), "event");
                TQ_CUDA(cudaEventSynchronize(e1[si]), "autotune sync");
                float t = 0;
                TQ_CUDA(cudaEventElapsedTime(&t, e0, e1[si]), "event time");
                ms = std::max(ms, t);
            }
            ms /= (float)(kReps * ns);
            sv->tune_ms[(size_t)b * nv + v] = ms;
            if (ms < best) {
                best = ms;
                sv->bucket_variant[b] = v;
            }
        }
        sv->bucket_ms[b] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1[0]);
    cudaEventDestroy(e1[1]);
    for (int si = 0; si < ns; ++si) {
        int herr = 0;
        TQ_CUDA(cudaMemcpy(&herr, sv->slots[si].d_err, sizeof(int), cudaMemcpyDeviceToHost), "D2H status");
        if (herr) return fail(TQ_ERR_TIMEOUT, "top-k kernel: a pipeline wait timed out (code %d)", herr);
    }
    if (fixed_variant < 0) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (int b = 0; b < nb; ++b)
            g_tune_cache[key_of(s0.bucket_rows[b])] = {sv->bucket_variant[b], sv->bucket_ms[b]};
    }
    return TQ_OK;
}

tq_status capture_graphs(tq_server *sv, Slot &sl) {
    for (size_t b = 0; b < sl.bucket_rows.size(); ++b) {
        cudaGraph_t g = nullptr;
        TQ_CUDA(cudaStreamBeginCapture(sl.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t e = enqueue_batch(sv, sl, sl.bucket_rows[b], sv->bucket_variant[b], true);
        cudaError_t e2 = cudaStreamEndCapture(sl.stream, &g);
        if (e != cudaSuccess) return cuda_fail(e, "capture batch");
        if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
        sl.graphs.push_back(ex);
    }
    return TQ_OK;
}

void finish_request(tq_server *sv, tq_request *r, double t) {
    {
        std::lock_guard<std::mutex> lk(r->mu);
        r->t_done = t;
        r->done = true;
    }
    r->cv.notify_all();
    const float lat = (float)(t - r->t_submit);
    if (sv->latencies_ms.size() < 1u << 20) {
        sv->latencies_ms.push_back(lat);
    } else {
        sv->latencies_ms[sv->lat_pos] = lat;
        sv->lat_pos = (sv->lat_pos + 1) % sv->latencies_ms.size();
    }
}

// The scheduler: completes finished batches, then packs queued requests into
// every free slot.
void worker_loop(tq_server *sv) {
    DeviceGuard g(sv->index->device);
    const int k = sv->k;
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        bool any_busy = false;
        for (auto &sl : sv->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) {
                any_busy = true;
                continue;
            }
            const double t = now_ms();
            const int herr = (q == cudaSuccess) ? *sl.h_err : 0;
            if (q == cudaSuccess) {
                sv->fallback_rows += (uint64_t)sl.h_cnt[tq::kCntFallbackRows];
                sv->bound_violations += (uint64_t)sl.h_cnt[tq::kCntBoundViolations];
                sv->scan_pass_rows += (uint64_t)sl.h_cnt[tq::kCntScanRows];
                sv->list_pass_rows += (uint64_t)sl.h_cnt[tq::kCntListRows];
            }
            size_t row = 0;
            for (tq_request *r : sl.batch) {
                if (q != cudaSuccess || herr) {
                    r->status = q != cudaSuccess ? TQ_ERR_CUDA : TQ_ERR_TIMEOUT;
                } else {
                    std::memcpy(r->dist.data(), sl.h_d + row * k, r->m * k * sizeof(float));
                    std::memcpy(r->idx.data(), sl.h_i + row * k, r->m * k * sizeof(long long));
                }
                row += r->m;
                release_request_rows(sv, r);
                finish_request(sv, r, t);
            }
            sv->completed += sl.batch.size();
            sv->rows_done += sl.batch_rows;
            sl.batch.clear();
            sl.batch_rows = 0;
            sl.busy = false;
        }
        if (sv->stop && sv->pending.empty() && !any_busy) break;
        for (auto &sl : sv->slots) {
            if (sl.busy || sv->pending.empty()) continue;
            size_t rows = 0;
            cudaError_t e = cudaSuccess;
            while (!sv->pending.empty() && rows + sv->pending.front()->m <= (size_t)sv->max_rows) {
                tq_request *r = sv->pending.front();
                sv->pending.pop_front();
                sv->pending_rows -= r->m;
                for (size_t i = 0; i < r->m; ++i) sl.h_rows[rows + i] = (int)(r->pool_off + i);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(sl.stream, r->uploaded, 0);
                rows += r->m;
                sl.batch.push_back(r);
            }
            if (sl.batch.empty()) continue;
            *sl.h_m = (int)rows;
            sl.batch_rows = rows;
            const int b = bucket_index(sv, rows);
            if (e == cudaSuccess) e = cudaGraphLaunch(sl.graphs[b], sl.stream);
            if (e == cudaSuccess) e = cudaEventRecord(sl.done, sl.stream);
            if (e != cudaSuccess) {
                for (tq_request *r : sl.batch) {
                    r->status = TQ_ERR_CUDA;
                    release_request_rows(sv, r);
                    finish_request(sv, r, now_ms());
                }
                sl.batch.clear();
                continue;
            }
            sl.busy = true;
            any_busy = true;
            ++sv->batches;
        }
        if (any_busy) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        } else {
            sv->cv.wait_for(lk, std::chrono::milliseconds(5),
                            [&] { return sv->stop || !sv->pending.empty(); });
        }
    }
}

}  // namespace

extern "C" {

tq_status tq_index_create_ex(const tq_space *csp, const uint8_t *codes, size_t n, int codes_on_device,
                             tq_index_layout layout, tq_index **out) {
    if (!out) return fail(TQ_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    tq_status st = tq::need_device(csp);
    if (st != TQ_OK) return st;
    if (n == 0 || !codes) return fail(TQ_ERR_INVALID_ARGUMENT, "index: empty corpus");
    if (n > 0x7ffffff0ull) return fail(TQ_ERR_INVALID_ARGUMENT, "index: more than 2^31 codes");
    if (layout != TQ_INDEX_PLANES && layout != TQ_INDEX_CODES)
        return fail(TQ_ERR_INVALID_ARGUMENT, "index: unknown layout %d", (int)layout);
    auto *sp = const_cast<tq_space *>(csp);
    const size_t K = 2 * sp->D;
    if (layout == TQ_INDEX_PLANES && K % 64)
        return fail(TQ_ERR_NOT_SUPPORTED, "index: padded dim must be a multiple of 32");
    if (layout == TQ_INDEX_CODES && (sp->D < 64 || sp->code_size % 4))
        return fail(TQ_ERR_NOT_SUPPORTED, "index: the codes layout needs a padded dim of at least 64");
    if (layout == TQ_INDEX_CODES && !tq::tc_topk_dec_ok(4, (int)sp->code_size))
        return fail(TQ_ERR_NOT_SUPPORTED,
                    "index: a tile of 128 codes of %zu bytes does not fit in shared memory; use the "
                    "planes layout", sp->code_size);
    DeviceGuard g(sp->device);
    auto *ix = new tq_index();
    ix->sp = sp;
    ix->n = n;
    ix->n_pad = round_up(n, 256);
    ix->K = (int)K;
    ix->layout = layout;
    ix->device = sp->device;
    for (float c : sp->centroids) ix->cmax = std::max(ix->cmax, std::fabs(c));
    const bool planes = layout == TQ_INDEX_PLANES;
    ix->K_lo = planes ? tq::asym_lo_width((int)sp->D) : 0;
    const size_t plane_bytes = planes ? ix->n_pad * (K + (size_t)ix->K_lo) * 2 : 0;
    const size_t code_bytes = round_up(n * sp->code_size, 256);
    const size_t nscal = planes ? 2 : 4;  // c1, c2 (+ fc, fs)
    cudaError_t e = cudaMalloc(&ix->block, plane_bytes + nscal * ix->n_pad * 4 + code_bytes +
                                               tq::kBoundFloats * 4 + 256);
    if (e != cudaSuccess) {
        delete ix;
        return cuda_fail(e, "cudaMalloc(index)");
    }
    auto *base = static_cast<unsigned char *>(ix->block);
    ix->planes = planes ? base : nullptr;
    ix->c1 = reinterpret_cast<float *>(base + plane_bytes);
    ix->c2 = ix->c1 + ix->n_pad;
    if (!planes) {
        ix->fc = ix->c2 + ix->n_pad;
        ix->fs = ix->fc + ix->n_pad;
    }
    ix->codes = reinterpret_cast<uint8_t *>(ix->c1 + nscal * ix->n_pad);
    ix->bound = reinterpret_cast<float *>(ix->codes + code_bytes);
    e = cudaMemcpy(ix->codes, codes, n * sp->code_size,
                   codes_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
    if (planes) {
        auto *hi = static_cast<unsigned char *>(ix->planes);
        auto *lo = hi + ix->n_pad * K * 2;
        const size_t chunk = 1 << 20;
        for (size_t r0 = 0; r0 < ix->n_pad && e == cudaSuccess; r0 += chunk) {
            const size_t rows_pad = std::min(chunk, ix->n_pad - r0);
            const size_t rows = r0 < n ? std::min(rows_pad, n - r0) : 0;
            e = tq::launch_planes_from_codes(sp->P, sp->T, ix->codes + std::min(r0, n - 1) * sp->code_size,
                                             rows, rows_pad, false, tq::kPlaneBF16, hi + r0 * K * 2,
                                             lo + r0 * (size_t)ix->K_lo * 2, ix->c1 + r0, ix->c2 + r0,
                                             nullptr);
        }
    } else if (e == cudaSuccess) {
        e = tq::launch_dec_factors(sp->P, ix->codes, n, ix->n_pad, false, ix->c1, ix->c2, ix->fc, ix->fs,
                                   nullptr);
    }
    if (e == cudaSuccess) e = tq::launch_index_bound(sp->P, ix->codes, n, ix->bound, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(ix->block);
        delete ix;
        return cuda_fail(e, "index build");
    }
    *out = ix;
    return TQ_OK;
}

tq_status tq_index_create(const tq_space *csp, const uint8_t *codes, size_t n, int codes_on_device,
                          tq_index **out) {
    return tq_index_create_ex(csp, codes, n, codes_on_device, TQ_INDEX_PLANES, out);
}

void tq_index_destroy(tq_index *ix) {
    if (!ix) return;
    DeviceGuard g(ix->device);
    if (ix->block) cudaFree(ix->block);
    delete ix;
}

tq_status tq_server_create_ex(tq_index *ix, const tq_server_params *prm, tq_server **out) {
    if (!out || !ix || !prm) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    const int k = prm->k, max_rows = prm->max_rows, kernel_variant = prm->kernel_variant;
    int slots = prm->slots;
    if (k < 1 || k > tq::kTopKMax) return fail(TQ_ERR_INVALID_ARGUMENT, "k must be in 1..%d", tq::kTopKMax);
    const int kc = prm->candidates ? prm->candidates : std::min(tq::kCandMax, k + 16);
    if (kc < k || kc > tq::kCandMax)
        return fail(TQ_ERR_INVALID_ARGUMENT, "candidates must be in k..%d", tq::kCandMax);
    if (!(prm->bound_scale >= 0.0f)) return fail(TQ_ERR_INVALID_ARGUMENT, "bound_scale must be >= 0");
    if (max_rows < 128 || max_rows % 128) return fail(TQ_ERR_INVALID_ARGUMENT, "max_rows must be a positive multiple of 128");
    if (slots < 1 || slots > 8) return fail(TQ_ERR_INVALID_ARGUMENT, "slots must be in 1..8");
    if (kernel_variant >= 0 && !variant_fits(ix, kernel_variant))
        return fail(TQ_ERR_INVALID_ARGUMENT, "kernel variant %d does not serve this index layout",
                    kernel_variant);
    DeviceGuard g(ix->device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
    if (max_rows / 128 > sms) return fail(TQ_ERR_INVALID_ARGUMENT, "max_rows too large for this GPU");
    auto *sv = new tq_server();
    sv->index = ix;
    sv->k = k;
    sv->kc = kc;
    sv->bound_scale = prm->bound_scale > 0.0f ? prm->bound_scale : 1.0f;
    sv->grid = sms;
    sv->fb_ctas = tq::fallback_ctas(sms);
    sv->max_rows = max_rows;
    sv->queue_rows_cap = prm->queue_rows ? prm->queue_rows : SIZE_MAX;
    // device memory: no more slots than fit in half the free memory; the
    // admission pool holds the queries of the queued and in-flight requests
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t dim = ix->sp->dim, row_bytes = dim * sizeof(float);
    const size_t budget = prm->memory_budget
                              ? prm->memory_budget
                              : std::min(free_b / 8, (size_t)16 * max_rows * row_bytes);
    sv->pool_rows = budget / row_bytes;
    if (sv->pool_rows < (size_t)max_rows) {
        delete sv;
        return fail(TQ_ERR_INVALID_ARGUMENT,
                    "memory budget of %zu bytes holds %zu query rows, fewer than max_rows (%d)",
                    budget, budget / row_bytes, max_rows);
    }
    const size_t D = ix->sp->D, K = (size_t)ix->K, R = (size_t)max_rows;
    const size_t slot_bytes =
        R * (ix->sp->dim * 4 + (2 * D + 2) * 4 + K * 4 + 8 + (size_t)k * 12 + (size_t)kc * 12 + 4 +
             (size_t)sv->fb_ctas * k * 8) +
        (size_t)sms * 128 * tq::kTopKListsMax * tq::kCandMax * 8 + 8192;
    const size_t fit = std::max<size_t>(1, (free_b / 2) / slot_bytes);
    slots = (int)std::min<size_t>((size_t)slots, fit);
    sv->slots.resize(slots);
    tq_status st = TQ_OK;
    cudaError_t ce = cudaMalloc(&sv->pool, sv->pool_rows * row_bytes);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&sv->up_stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) st = cuda_fail(ce, "admission pool");
    sv->pool_free.emplace(0, sv->pool_rows);
    for (auto &sl : sv->slots)
        if (st == TQ_OK && (st = slot_alloc(sv, sl)) != TQ_OK) break;
    if (st == TQ_OK) st = autotune(sv, kernel_variant);
    for (auto &sl : sv->slots) {
        if (st != TQ_OK) break;
        st = capture_graphs(sv, sl);
    }
    if (st != TQ_OK) {
        for (auto &sl : sv->slots) slot_free(sl);
        if (sv->pool) cudaFree(sv->pool);
        if (sv->up_stream) cudaStreamDestroy(sv->up_stream);
        delete sv;
        return st;
    }
    sv->worker = std::thread(worker_loop, sv);
    *out = sv;
    return TQ_OK;
}

tq_status tq_server_create(tq_index *ix, int k, int max_rows, int slots, int kernel_variant,
                           size_t queue_rows, tq_server **out) {
    tq_server_params p{};
    p.k = k;
    p.max_rows = max_rows;
    p.slots = slots;
    p.kernel_variant = kernel_variant;
    p.queue_rows = queue_rows;
    return tq_server_create_ex(ix, &p, out);
}

tq_status tq_server_submit(tq_server *sv, const float *queries, size_t m, tq_request **out) {
    if (!sv || !out || (m && !queries)) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (m == 0 || m > (size_t)sv->max_rows)
        return fail(TQ_ERR_INVALID_ARGUMENT, "request rows must be in 1..%d", sv->max_rows);
    if (m > sv->pool_rows)
        return fail(TQ_ERR_INVALID_ARGUMENT, "request of %zu rows exceeds the admission pool (%zu rows)",
                    m, sv->pool_rows);
    const size_t dim = sv->index->sp->dim;
    auto *r = new tq_request();
    r->queries.assign(queries, queries + m * dim);
    r->m = m;
    r->k = sv->k;
    r->dist.assign(m * sv->k, 0.0f);
    r->idx.assign(m * sv->k, -1);
    r->t_submit = now_ms();
    {
        // admission: room in the pool (and under the optional queued-row cap)
        std::lock_guard<std::mutex> lk(sv->mu);
        ++sv->submitted;
        if (sv->stop || sv->pending_rows + m > sv->queue_rows_cap || !pool_alloc(sv, m, &r->pool_off)) {
            ++sv->rejected;
            const size_t used = sv->pool_used, queued = sv->pending_rows;
            delete r;
            return fail(TQ_ERR_BUSY, "admission refused: %zu of %zu pool rows in use, %zu rows queued",
                        used, sv->pool_rows, queued);
        }
    }
    // the queries go to their pool rows now; the batch that takes them waits
    // for this copy on the device
    DeviceGuard g(sv->index->device);
    cudaError_t e = cudaEventCreateWithFlags(&r->uploaded, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sv->pool + r->pool_off * dim, r->queries.data(), m * dim * sizeof(float),
                            cudaMemcpyHostToDevice, sv->up_stream);
    if (e == cudaSuccess) e = cudaEventRecord(r->uploaded, sv->up_stream);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (e != cudaSuccess) {
            release_request_rows(sv, r);
            delete r;
            return cuda_fail(e, "request upload");
        }
        sv->pending.push_back(r);
        sv->pending_rows += m;
    }
    sv->cv.notify_one();
    *out = r;
    return TQ_OK;
}

tq_status tq_request_wait(tq_request *r, int timeout_ms, float *dist, int64_t *idx,
                          double *latency_ms) {
    if (!r) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL request");
    std::unique_lock<std::mutex> lk(r->mu);
    if (timeout_ms < 0) {
        r->cv.wait(lk, [&] { return r->done; });
    } else if (!r->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; })) {
        return fail(TQ_ERR_TIMEOUT, "request not finished within %d ms", timeout_ms);
    }
    if (r->status != TQ_OK) return fail(r->status, "request failed on the device");
    if (dist) std::memcpy(dist, r->dist.data(), r->dist.size() * sizeof(float));
    if (idx) std::memcpy(idx, r->idx.data(), r->idx.size() * sizeof(long long));
    if (latency_ms) *latency_ms = r->t_done - r->t_submit;
    return TQ_OK;
}

int tq_request_done(tq_request *r) {
    if (!r) return 0;
    std::lock_guard<std::mutex> lk(r->mu);
    return r->done ? 1 : 0;
}

void tq_request_release(tq_request *r) {
    if (!r) return;
    {
        std::unique_lock<std::mutex> lk(r->mu);
        r->cv.wait(lk, [&] { return r->done; });
    }
    delete r;
}

tq_status tq_server_get_stats(tq_server *sv, tq_server_stats *out, float *latencies, size_t cap,
                          size_t *n_lat) {
    if (!sv || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    out->submitted = sv->submitted;
    out->rejected = sv->rejected;
    out->completed = sv->completed;
    out->batches = sv->batches;
    out->rows = sv->rows_done;
    out->queued_rows = sv->pending_rows;
    out->slots = (int)sv->slots.size();
    out->max_rows = sv->max_rows;
    out->candidates = sv->kc;
    out->fallback_rows = sv->fallback_rows;
    out->bound_violations = sv->bound_violations;
    out->scan_pass_rows = sv->scan_pass_rows;
    out->list_pass_rows = sv->list_pass_rows;
    out->pool_rows = sv->pool_rows;
    out->pool_used_rows = sv->pool_used;
    size_t nl = std::min(cap, sv->latencies_ms.size());
    if (latencies && nl) std::memcpy(latencies, sv->latencies_ms.data(), nl * sizeof(float));
    if (n_lat) *n_lat = latencies ? nl : sv->latencies_ms.size();
    return TQ_OK;
}

tq_status tq_server_reset_stats(tq_server *sv) {
    if (!sv) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->submitted = sv->rejected = sv->completed = sv->batches = sv->rows_done = 0;
    sv->fallback_rows = sv->bound_violations = sv->scan_pass_rows = sv->list_pass_rows = 0;
    sv->latencies_ms.clear();
    sv->lat_pos = 0;
    return TQ_OK;
}

tq_status tq_server_tuning(tq_server *sv, int *bucket_rows, int *variant, float *ms, int cap, int *n) {
    if (!sv) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL server");
    const auto &b = sv->slots[0].bucket_rows;
    const int nb = (int)std::min<size_t>(b.size(), (size_t)cap);
    for (int i = 0; i < nb; ++i) {
        if (bucket_rows) bucket_rows[i] = b[i];
        if (variant) variant[i] = sv->bucket_variant[i];
        if (ms) ms[i] = (float)sv->bucket_ms[i];
    }
    if (n) *n = (int)b.size();
    return TQ_OK;
}

tq_status tq_server_tuning_times(tq_server *sv, float *ms, int cap, int *n_buckets,
                                 int *n_variants, int *from_cache) {
    if (!sv) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL server");
    const int nb = (int)sv->slots[0].bucket_rows.size(), nv = tq::tc_topk_variants();
    if (ms) {
        const int c = std::min(cap, nb * nv);
        for (int i = 0; i < c; ++i) ms[i] = sv->tune_ms.empty() ? 0.0f : sv->tune_ms[(size_t)i];
    }
    if (n_buckets) *n_buckets = nb;
    if (n_variants) *n_variants = nv;
    if (from_cache) *from_cache = sv->tuned_from_cache ? 1 : 0;
    return TQ_OK;
}

tq_status tq_topk_variant_shape(int variant, int *shape) {
    int v[4];
    if (!shape || !tq::tc_topk_shape(variant, v))
        return fail(TQ_ERR_INVALID_ARGUMENT, "unknown kernel variant %d", variant);
    for (int i = 0; i < 4; ++i) shape[i] = v[i];
    return TQ_OK;
}

tq_status tq_selftest_bounded_wait(int device, int budget_ms) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TQ_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0) cudaGetDevice(&device);
    if (budget_ms < 1 || budget_ms > 10000) return fail(TQ_ERR_INVALID_ARGUMENT, "budget_ms must be in 1..10000");
    DeviceGuard g(device);
    int clock_khz = 0;
    cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, device);
    if (clock_khz <= 0) clock_khz = 2000000;
    int *err = nullptr;
    TQ_CUDA(cudaMalloc(&err, sizeof(int)), "cudaMalloc");
    cudaError_t e = cudaMemset(err, 0, sizeof(int));
    if (e == cudaSuccess) e = tq::launch_bounded_wait_selftest(err, (long long)clock_khz * budget_ms, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(err);
    if (e != cudaSuccess) return cuda_fail(e, "bounded-wait self-test");
    if (h != 0) return fail(TQ_ERR_TIMEOUT, "device wait gave up after ~%d ms (code %d)", budget_ms, h);
    return TQ_OK;
}

void tq_server_destroy(tq_server *sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    DeviceGuard g(sv->index->device);
    for (auto &sl : sv->slots) slot_free(sl);
    if (sv->up_stream) {
        cudaStreamSynchronize(sv->up_stream);
        cudaStreamDestroy(sv->up_stream);
    }
    if (sv->pool) cudaFree(sv->pool);
    delete sv;
}

}  // extern "C"
