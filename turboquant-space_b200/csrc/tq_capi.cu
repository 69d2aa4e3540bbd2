// tq_capi.cu -- the C ABI (include/turboquant_b200.h) over the sm_100a kernels.
//
// Host responsibilities: argument validation (the reference binding's checks,
// python/turboquant/bindings.cpp:14-49, 159-209), table construction and
// upload, device selection, stream-ordered scratch, and chunked host<->device
// streaming for the host-pointer entry points.  No C++ exception crosses the
// ABI: every entry point catches and converts to a tq_status.
#include "turboquant_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "tq_exact.h"
#include "tq_host.h"
#include "tq_internal.h"
#include "tq_mton.h"
#include "tq_tables.h"


thread_local std::string g_err;

namespace tq {

tq_status fail(tq_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

tq_status cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(TQ_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(TQ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

tq_status need_device(const tq_space *sp) {
    if (!sp) return fail(TQ_ERR_INVALID_ARGUMENT, "space is NULL");
    if (sp->device < 0 || !sp->dev_block)
        return fail(TQ_ERR_NO_DEVICE,
                    "no CUDA device: the TurboQuant B200 kernels need an sm_100 GPU");
    return TQ_OK;
}

}  // namespace tq

using tq::cuda_fail;
using tq::DeviceGuard;
using tq::fail;
using tq::need_device;

namespace {

int ilog2(size_t v) {
    int l = 0;
    while ((size_t(1) << l) < v) ++l;
    return l;
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

tq_status check_dev(const void *p, size_t bytes, const char *name) {
    if (bytes == 0) return TQ_OK;
    if (!p) return fail(TQ_ERR_INVALID_ARGUMENT, "%s: NULL pointer", name);
    if (!is_device_ptr(p)) return fail(TQ_ERR_INVALID_ARGUMENT, "%s: not a device pointer", name);
    return TQ_OK;
}

// Reads and clears the space's device status word (after the caller's
// synchronisation); TQ_ERR_TIMEOUT when a bounded device wait gave up.
tq_status take_status(const tq_space *sp, int *code_out) {
    int code = 0;
    TQ_CUDA(cudaMemcpy(&code, sp->T.status, sizeof(int), cudaMemcpyDeviceToHost), "read status");
    if (code_out) *code_out = code;
    if (code == 0) return TQ_OK;
    TQ_CUDA(cudaMemset(sp->T.status, 0, sizeof(int)), "clear status");
    return fail(TQ_ERR_TIMEOUT, "a bounded device-side wait gave up (code %d)", code);
}

tq_status check_codes_align(const void *p, const char *name) {
    if (reinterpret_cast<uintptr_t>(p) & 3)
        return fail(TQ_ERR_INVALID_ARGUMENT, "%s: device codes must be 4-byte aligned", name);
    return TQ_OK;
}

// Stream-ordered scratch from the device's default pool.
struct Scratch {
    void *p = nullptr;
    cudaStream_t st = nullptr;
    ~Scratch() {
        if (p) cudaFreeAsync(p, st);
    }
    cudaError_t alloc(size_t bytes, cudaStream_t s) {
        st = s;
        return cudaMallocAsync(&p, bytes, s);
    }
};

constexpr size_t kChunkBytes = size_t(256) << 20;  // host streaming granularity

tq_status ensure_host_streams(tq_space *sp) {
    for (auto &s : sp->host_stream)
        if (!s) TQ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    return TQ_OK;
}

// Precisions of the M x N entry points: FP32, split-BF16 (planes or decoded
// tiles) and the reference-order arithmetic, for both forms.
tq_status mton_precision_ok(tq_precision p, bool sym) {
    if (p == TQ_PRECISION_FP32 || p == TQ_PRECISION_SPLIT_BF16 || p == TQ_PRECISION_SPLIT_BF16_DECODED ||
        p == TQ_PRECISION_REFERENCE)
        return TQ_OK;
    if (p == TQ_PRECISION_SPLIT_TF32)
        return fail(TQ_ERR_NOT_SUPPORTED, "precision %d is not available for %s distances", (int)p,
                    sym ? "symmetric" : "asymmetric");
    return fail(TQ_ERR_INVALID_ARGUMENT, "unknown precision %d", (int)p);
}

// M x N driver.  The row side (m queries, or m codes for the symmetric form)
// is prepared once; the column side is decoded and contracted in chunks:
//   FP32, m < kScanRows:  the HBM-bound scan kernel per row (no planes);
//   FP32 otherwise:       FP32 planes + CUDA-core SGEMM;
//   SPLIT_BF16:           hi/lo BF16 planes + tcgen05 GEMM;
//   SPLIT_BF16_DECODED:   the same row planes; the column tiles decoded from the
//                         codes in shared memory (per-code scalars only in HBM);
//   REFERENCE:            the reference build's own arithmetic, one pair per thread.
// Every distance ends in the same epilogue d = max(0, r2 + c2 - 2 C r1 c1).
class MtonRunner {
  public:
    static constexpr size_t kScanRows = 32;
    static constexpr size_t kRowPlaneBytes = size_t(512) << 20;
    static constexpr size_t kColPlaneBytes = size_t(1) << 30;

    static size_t row_chunk(const tq_space *sp, bool sym, tq_precision prec) {
        const size_t K = sym ? sp->D : 2 * sp->D;
        size_t rows = (kRowPlaneBytes / (K * 4)) & ~size_t(tq::kPlaneRowAlign - 1);
        (void)prec;
        return std::max<size_t>(tq::kPlaneRowAlign, rows);
    }

    MtonRunner(tq_space *sp, bool sym, tq_precision prec, size_t m)
        : sp_(sp), sym_(sym), prec_(prec), m_(m) {
        K_ = sym ? (int)sp->D : 2 * (int)sp->D;
        dec_ = prec == TQ_PRECISION_SPLIT_BF16_DECODED;
        fmt_ = (prec == TQ_PRECISION_SPLIT_BF16 || dec_) ? tq::kPlaneBF16 : tq::kPlaneF32;
        planes_ = prec != TQ_PRECISION_REFERENCE &&
                  (prec == TQ_PRECISION_SPLIT_BF16 || dec_ || m >= kScanRows);
        m_pad_ = round_up(m, tq::kPlaneRowAlign);
        const size_t col_align = prec == TQ_PRECISION_SPLIT_BF16 ? 256 : 128;
        nc_max_ = std::max(col_align, ((kColPlaneBytes / ((size_t)K_ * 4)) / col_align) * col_align);
    }

    tq_status prepare_rows(const void *rows_dev, cudaStream_t s) {
        if (prec_ == TQ_PRECISION_SPLIT_BF16 && (K_ % 64 != 0))
            return fail(TQ_ERR_NOT_SUPPORTED,
                        "split-BF16 contraction needs a reduction length that is a multiple of 64 "
                        "(padded dim %zu)", sp_->D);
        if (dec_ && sp_->D % 64 != 0)
            return fail(TQ_ERR_NOT_SUPPORTED,
                        "decoded split-BF16 tiles need a padded dim that is a multiple of 64 (padded dim %zu)",
                        sp_->D);
        if (dec_ && !tq::tc_dist_dec_fits((int)sp_->code_size))
            return fail(TQ_ERR_NOT_SUPPORTED,
                        "decoded split-BF16 tiles: a tile of 128 codes of %zu bytes does not fit in shared "
                        "memory beside the pipeline (use split_bf16)", sp_->code_size);
        if (fmt_ == tq::kPlaneF32 && planes_ && (K_ % 16 != 0)) planes_ = false;
        const size_t D = sp_->D;
        if (!sym_) {  // prepared queries (the scan path uses them directly)
            TQ_CUDA(prep_.alloc(sizeof(float) * m_ * (2 * D + 2), s), "cudaMallocAsync(prepared)");
            q_rot_ = static_cast<float *>(prep_.p);
            s_q_ = q_rot_ + m_ * D;
            norms_ = s_q_ + m_ * D;
            TQ_CUDA(tq::launch_prepare(sp_->P, sp_->T, static_cast<const float *>(rows_dev), m_,
                                       q_rot_, s_q_, norms_, s),
                    "prepare kernel");
        } else {
            codes_a_ = static_cast<const uint8_t *>(rows_dev);
        }
        if (!planes_) return TQ_OK;
        const size_t plane_bytes = m_pad_ * (size_t)K_ * 4;
        TQ_CUDA(rows_.alloc(plane_bytes + 2 * 4 * m_pad_, s), "cudaMallocAsync(row planes)");
        a0_ = rows_.p;
        a1_ = static_cast<unsigned char *>(rows_.p) + plane_bytes / 2;
        r1_ = reinterpret_cast<float *>(static_cast<unsigned char *>(rows_.p) + plane_bytes);
        r2_ = r1_ + m_pad_;
        if (!sym_)
            TQ_CUDA(tq::launch_planes_from_prepared(q_rot_, s_q_, norms_, m_, m_pad_, (int)D, fmt_, a0_,
                                                    a1_, r1_, r2_, s),
                    "row planes");
        else
            TQ_CUDA(tq::launch_planes_from_codes(sp_->P, sp_->T, codes_a_, m_, m_pad_, true, fmt_, a0_,
                                                 a1_, r1_, r2_, s),
                    "row planes");
        return TQ_OK;
    }

    // columns [0, n) of device codes -> out[i * ldo + j]
    tq_status run_cols(const uint8_t *codes, size_t n, float *out, size_t ldo, cudaStream_t s) {
        if (dec_) return run_cols_decoded(codes, n, out, ldo, s);
        if (!planes_) {
            if (!sym_ && prec_ == TQ_PRECISION_REFERENCE)
                TQ_CUDA(tq::launch_exact_mton(sp_->P, sp_->T.centroids, q_rot_, s_q_, norms_, m_, codes,
                                              n, out, ldo, s),
                        "reference-order m_to_n kernel");
            else if (!sym_)
                TQ_CUDA(tq::launch_mton_fp32(sp_->P, sp_->T, q_rot_, s_q_, norms_, m_, codes, n, out,
                                             ldo, s),
                        "m_to_n scan kernel");
            else if (prec_ == TQ_PRECISION_REFERENCE)
                TQ_CUDA(tq::launch_exact_mton_sym(sp_->P, sp_->T.centroids, codes_a_, m_, codes, n, out,
                                                  ldo, s),
                        "reference-order symmetric m_to_n kernel");
            else
                TQ_CUDA(tq::launch_mton_sym_fp32(sp_->P, sp_->T, codes_a_, m_, codes, n, out, ldo, s),
                        "symmetric m_to_n scan kernel");
            return TQ_OK;
        }
        if (!cols_.p) {
            const size_t nc = std::min(nc_max_, round_up(n, prec_ == TQ_PRECISION_SPLIT_BF16 ? 256 : 128));
            nc_alloc_ = nc;
            const size_t plane_bytes = nc * (size_t)K_ * 4;
            TQ_CUDA(cols_.alloc(plane_bytes + 2 * 4 * nc + 16, s), "cudaMallocAsync(column planes)");
            b0_ = cols_.p;
            b1_ = static_cast<unsigned char *>(cols_.p) + plane_bytes / 2;
            c1_ = reinterpret_cast<float *>(static_cast<unsigned char *>(cols_.p) + plane_bytes);
            c2_ = c1_ + nc;
            err_ = reinterpret_cast<int *>(c2_ + nc);
            TQ_CUDA(cudaMemsetAsync(err_, 0, sizeof(int), s), "memset");
        }
        const size_t col_align = prec_ == TQ_PRECISION_SPLIT_BF16 ? 256 : 128;
        for (size_t n0 = 0; n0 < n; n0 += nc_alloc_) {
            const size_t nc = std::min(nc_alloc_, n - n0);
            const size_t nc_pad = round_up(nc, col_align);
            TQ_CUDA(tq::launch_planes_from_codes(sp_->P, sp_->T, codes + n0 * sp_->code_size, nc,
                                                 nc_pad, sym_, fmt_, b0_, b1_, c1_, c2_, s),
                    "column planes");
            if (fmt_ == tq::kPlaneF32)
                TQ_CUDA(tq::launch_sgemm_dist(static_cast<const float *>(a0_),
                                              static_cast<const float *>(b0_), K_, m_, m_pad_, nc,
                                              nc_pad, r1_, r2_, c1_, c2_, out + n0, ldo, s),
                        "FP32 GEMM kernel");
            else
                TQ_CUDA(tq::launch_tc_dist(a0_, a1_, b0_, b1_, K_,
                                           sym_ ? K_ : tq::asym_lo_width((int)sp_->D), m_, m_pad_,
                                           nc, nc_pad, r1_, r2_, c1_, c2_, out + n0, ldo, err_, s),
                        "tcgen05 GEMM kernel");
        }
        return TQ_OK;
    }

    // The decoded form: per chunk of columns, the per-code scalars (16 bytes a
    // code) and one tensor-core launch whose decoder warps turn each tile of 128
    // codes into its B tiles in shared memory.  A tile's codes arrive by one bulk
    // copy rounded up to 16 bytes; whole tiles are multiples of 16 bytes, and a
    // ragged last tile whose bytes do not end on that boundary is read from a
    // padded copy, so no copy reads past the caller's codes.
    tq_status run_cols_decoded(const uint8_t *codes, size_t n, float *out, size_t ldo, cudaStream_t s) {
        const size_t cs = sp_->code_size;
        if (reinterpret_cast<uintptr_t>(codes) & 15)
            return fail(TQ_ERR_NOT_SUPPORTED, "decoded split-BF16 tiles need 16-byte aligned device codes");
        if (!cols_.p) {
            nc_alloc_ = std::min(round_up(n, 128), kDecCols);
            tail_bytes_ = round_up(128 * cs, 16) + 16;
            TQ_CUDA(cols_.alloc(4 * 4 * nc_alloc_ + 16 + tail_bytes_, s), "cudaMallocAsync(column scalars)");
            c1_ = static_cast<float *>(cols_.p);
            c2_ = c1_ + nc_alloc_;
            fc_ = c2_ + nc_alloc_;
            fs_ = fc_ + nc_alloc_;
            err_ = reinterpret_cast<int *>(fs_ + nc_alloc_);
            tail_ = reinterpret_cast<uint8_t *>(err_ + 4);
            TQ_CUDA(cudaMemsetAsync(err_, 0, sizeof(int), s), "memset");
        }
        tq::DecSrc d;
        d.cs = (int)cs;
        d.nibble = sp_->P.nibble;
        d.kbc = (int)(sp_->D / 64);
        d.centroids = sp_->T.centroids;
        d.levels = (int)sp_->levels;
        auto launch = [&](const uint8_t *src, size_t cols, float *dst) -> tq_status {
            const size_t cols_pad = round_up(cols, 128);
            TQ_CUDA(tq::launch_dec_factors(sp_->P, src, cols, cols_pad, sym_, c1_, c2_, sym_ ? nullptr : fc_,
                                           sym_ ? nullptr : fs_, s),
                    "column scalars");
            d.codes = src;
            d.n = (unsigned)cols;
            d.fc = sym_ ? nullptr : fc_;
            d.fs = sym_ ? nullptr : fs_;
            TQ_CUDA(tq::launch_tc_dist_dec(a0_, a1_, m_, m_pad_, d, cols_pad, K_, r1_, r2_, c1_, c2_, dst, ldo,
                                           err_, s),
                    "tcgen05 GEMM kernel (decoded tiles)");
            return TQ_OK;
        };
        for (size_t n0 = 0; n0 < n; n0 += nc_alloc_) {
            const size_t nc = std::min(nc_alloc_, n - n0);
            const size_t rem = nc % 128;
            const size_t n_main = (rem != 0 && (rem * cs) % 16 != 0) ? nc - rem : nc;
            tq_status st;
            if (n_main > 0 && (st = launch(codes + n0 * cs, n_main, out + n0)) != TQ_OK) return st;
            if (n_main < nc) {
                TQ_CUDA(cudaMemcpyAsync(tail_, codes + (n0 + n_main) * cs, (nc - n_main) * cs,
                                        cudaMemcpyDeviceToDevice, s),
                        "copy of the last tile");
                if ((st = launch(tail_, nc - n_main, out + n0 + n_main)) != TQ_OK) return st;
            }
        }
        return TQ_OK;
    }

    // Reports a bounded wait that gave up inside the tensor-core kernel.
    tq_status finish(cudaStream_t s) {
        if (!err_) return TQ_OK;
        int h = 0;
        TQ_CUDA(cudaMemcpyAsync(&h, err_, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H status");
        TQ_CUDA(cudaStreamSynchronize(s), "sync");
        if (h != 0) return fail(TQ_ERR_TIMEOUT, "tensor-core kernel: a pipeline wait timed out (code %d)", h);
        return TQ_OK;
    }

  private:
    static constexpr size_t kDecCols = size_t(1) << 24;  // columns per decoded launch
    static size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
    tq_space *sp_;
    bool sym_, dec_ = false;
    size_t tail_bytes_ = 0;
    float *fc_ = nullptr, *fs_ = nullptr;
    uint8_t *tail_ = nullptr;
    tq_precision prec_;
    size_t m_, m_pad_ = 0, nc_max_ = 0, nc_alloc_ = 0;
    int K_ = 0, fmt_ = 0;
    bool planes_ = false;
    Scratch prep_, rows_, cols_;
    float *q_rot_ = nullptr, *s_q_ = nullptr, *norms_ = nullptr;
    const uint8_t *codes_a_ = nullptr;
    void *a0_ = nullptr, *a1_ = nullptr, *b0_ = nullptr, *b1_ = nullptr;
    float *r1_ = nullptr, *r2_ = nullptr, *c1_ = nullptr, *c2_ = nullptr;
    int *err_ = nullptr;
};

}  // namespace

extern "C" {

const char *tq_last_error(void) { return g_err.c_str(); }
const char *tq_version(void) { return "turboquant-b200 0.1.0 (sm_100a)"; }

tq_status tq_space_create(size_t dim, int bits, uint64_t rot_seed, uint64_t qjl_seed,
                          int num_threads, int device, tq_space **out) {
    if (!out) return fail(TQ_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (dim < 1) return fail(TQ_ERR_INVALID_ARGUMENT, "TurboQuantSpace: dim must be >= 1");
    if (bits < 2)
        return fail(TQ_ERR_INVALID_ARGUMENT,
                    "TurboQuantSpace: need at least 2 bits (1 MSE + 1 QJL)");
    if (bits > 9)
        return fail(TQ_ERR_INVALID_ARGUMENT, "TurboQuantSpace: max 9 bits (8-bit MSE + 1 QJL)");
    try {
        auto *sp = new tq_space();
        sp->dim = dim;
        size_t D = 1;
        while (D < (dim < 4 ? 4 : dim)) D <<= 1;  // roundUpPow2(max(dim, 4)) :233-238, 258
        const int log2D = ilog2(D);
        if (log2D > tq::kMaxLogD) {
            delete sp;
            return fail(TQ_ERR_NOT_SUPPORTED,
                        "TurboQuantSpace: padded dim %zu exceeds the supported maximum %d", D,
                        1 << tq::kMaxLogD);
        }
        sp->D = D;
        sp->padded = D != dim;
        sp->bits = bits;
        sp->packed_bytes = bits <= 4 ? (D + 1) / 2 : D;  // turbo_quant.h:177-179
        sp->code_size = sp->packed_bytes + 12;            // :182-184
        sp->levels = 1 << (bits - 1);
        sp->rot_seed = rot_seed;
        sp->qjl_seed = qjl_seed;
        sp->num_threads = num_threads > 0 ? num_threads : 1;
        if (sp->padded)  // the reference's warning, space_turbo_quant.h:269-273
            fprintf(stderr,
                    "[TurboQuantSpace] warning: input dim %zu is not a power of 2 (or < 4); "
                    "padding to %zu with zeros for internal computation.\n",
                    dim, D);
        tq::lloyd_max(bits - 1, sp->centroids, sp->boundaries);
        sp->rot_signs = tq::sign_vector(D, rot_seed);
        sp->qjl_signs = tq::sign_vector(D, qjl_seed);

        tq::Params &P = sp->P;
        P.dim = (int)dim;
        P.D = (int)D;
        P.log2D = log2D;
        P.bits = bits;
        P.nibble = bits <= 4;
        P.levels = sp->levels;
        P.nb = sp->levels - 1;
        P.pb = (int)sp->packed_bytes;
        P.cs = (int)sp->code_size;
        // space_turbo_quant.h:265-266 and turbo_quant.h:69, in FP32 as written
        P.scale = std::sqrt(static_cast<float>(M_PI) / 2.0f) / std::sqrt(static_cast<float>(D));
        P.wht_scale = 1.0f / std::sqrt(static_cast<float>(D));
        P.lutq = 0;
        P.qlut_k = 0;
        P.qflag = 0;
        if (tq::build_quant_lut(sp->boundaries, tq::kQlutBuckets, tq::kQlutMaxK, sp->qlut)) {
            P.lutq = 1;
            P.qlut_k = sp->qlut.k;
            P.qlut_s = sp->qlut.s;
            P.qlut_c = sp->qlut.c;
            // one boundary at most per bucket and lo < 128: bit 7 can flag the
            // buckets that hold one (the others need no comparison)
            P.qflag = (P.qlut_k == 1 && sp->levels <= 128) ? 1 : 0;
        }

        // device binding (optional: without a GPU the space answers geometry
        // and table queries, and every compute entry point reports NO_DEVICE)
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
            cudaGetLastError();
            ndev = 0;
        }
        if (ndev > 0) {
            int dev = device;
            if (dev < 0) cudaGetDevice(&dev);
            if (dev >= ndev) {
                delete sp;
                return fail(TQ_ERR_INVALID_ARGUMENT, "device %d out of range (%d devices)", dev, ndev);
            }
            int major = 0;
            cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
            if (major != 10) {
                delete sp;
                return fail(TQ_ERR_NO_DEVICE, "device %d is sm_%d*, these kernels are built for sm_100a",
                            dev, major);
            }
            DeviceGuard g(dev);
            const size_t mw = (D + 31) / 32;
            const size_t off_c = 0, off_b = 4 * 256, off_q = off_b + 4 * (256 + tq::kQlutMaxK + 4);
            const size_t off_qf = off_q + tq::kQlutBuckets;
            const size_t off_r = off_qf + tq::kQlutBuckets, off_j = off_r + 4 * mw;
            const size_t off_s = (off_j + 4 * mw + 15) & ~size_t(15);
            const size_t total = off_s + 16;
            std::vector<unsigned char> host(total, 0);
            std::memcpy(host.data() + off_c, sp->centroids.data(), 4 * sp->levels);
            std::vector<float> bnd(256 + tq::kQlutMaxK + 4, INFINITY);
            std::copy(sp->boundaries.begin(), sp->boundaries.end(), bnd.begin());
            std::memcpy(host.data() + off_b, bnd.data(), 4 * bnd.size());
            if (P.lutq) {
                std::memcpy(host.data() + off_q, sp->qlut.lo.data(), tq::kQlutBuckets);
                for (int j = 0; j < tq::kQlutBuckets; ++j)
                    host[off_qf + j] = (uint8_t)(sp->qlut.lo[j] | ((P.qflag && sp->qlut.span[j]) ? 0x80 : 0));
            }
            std::vector<uint32_t> rm(mw, 0), qm(mw, 0);
            for (size_t i = 0; i < D; ++i) {
                if (sp->rot_signs[i] > 0) rm[i >> 5] |= 1u << (i & 31);
                if (sp->qjl_signs[i] > 0) qm[i >> 5] |= 1u << (i & 31);
            }
            std::memcpy(host.data() + off_r, rm.data(), 4 * mw);
            std::memcpy(host.data() + off_j, qm.data(), 4 * mw);
            cudaError_t e = cudaMalloc(&sp->dev_block, total);
            if (e != cudaSuccess) {
                delete sp;
                return cuda_fail(e, "cudaMalloc(tables)");
            }
            e = cudaMemcpy(sp->dev_block, host.data(), total, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(sp->dev_block);
                delete sp;
                return cuda_fail(e, "cudaMemcpy(tables)");
            }
            auto *base = static_cast<unsigned char *>(sp->dev_block);
            sp->T.centroids = reinterpret_cast<const float *>(base + off_c);
            sp->T.boundaries = reinterpret_cast<const float *>(base + off_b);
            sp->T.qlut = base + off_q;
            sp->T.qlutf = base + off_qf;
            sp->T.rot_mask = reinterpret_cast<const uint32_t *>(base + off_r);
            sp->T.qjl_mask = reinterpret_cast<const uint32_t *>(base + off_j);
            sp->T.status = reinterpret_cast<int *>(base + off_s);
            sp->device = dev;
            // keep freed scratch in the pool between calls
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t thr = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            }
        }
        *out = sp;
        return TQ_OK;
    } catch (const std::bad_alloc &) {
        return fail(TQ_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        return fail(TQ_ERR_CUDA, "unexpected failure in tq_space_create");
    }
}

void tq_space_destroy(tq_space *sp) {
    if (!sp) return;
    if (sp->device >= 0) {
        DeviceGuard g(sp->device);
        for (auto &s : sp->host_stream)
            if (s) cudaStreamDestroy(s);
        for (auto e : sp->timer_events) cudaEventDestroy(e);
        if (sp->dev_block) cudaFree(sp->dev_block);
    }
    delete sp;
}

tq_status tq_space_get_info(const tq_space *sp, tq_space_info *info) {
    if (!sp || !info) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL argument");
    info->dim = sp->dim;
    info->padded_dim = sp->D;
    info->packed_bytes = sp->packed_bytes;
    info->code_size = sp->code_size;
    info->bits_per_coord = sp->bits;
    info->num_levels = sp->levels;
    info->padded = sp->padded ? 1 : 0;
    info->num_threads = sp->num_threads;
    info->device = sp->device;
    info->rot_seed = sp->rot_seed;
    info->qjl_seed = sp->qjl_seed;
    info->scale = sp->P.scale;
    return TQ_OK;
}

tq_status tq_space_tables(const tq_space *sp, float *centroids, float *boundaries,
                          float *rot_signs, float *qjl_signs) {
    if (!sp) return fail(TQ_ERR_INVALID_ARGUMENT, "space is NULL");
    if (centroids) std::memcpy(centroids, sp->centroids.data(), 4 * sp->centroids.size());
    if (boundaries) std::memcpy(boundaries, sp->boundaries.data(), 4 * sp->boundaries.size());
    if (rot_signs) std::memcpy(rot_signs, sp->rot_signs.data(), 4 * sp->rot_signs.size());
    if (qjl_signs) std::memcpy(qjl_signs, sp->qjl_signs.data(), 4 * sp->qjl_signs.size());
    return TQ_OK;
}

tq_status tq_space_quantize(const tq_space *sp, const float *z, size_t n, uint8_t *idx) {
    if (!sp) return fail(TQ_ERR_INVALID_ARGUMENT, "space is NULL");
    if (n && (!z || !idx)) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    const tq::Params &P = sp->P;
    for (size_t i = 0; i < n; ++i) {
        int c = 0;
        if (P.lutq) {
            const int j = tq::quant_bucket(z[i], P.qlut_s, P.qlut_c, tq::kQlutBuckets);
            c = sp->qlut.lo[j];
            const int lo = c;
            // as the encode kernel's flagged table (P.qflag): a bucket that holds
            // no boundary takes lo without a comparison
            const int kc = (P.qflag && sp->qlut.span[j] == 0) ? 0 : P.qlut_k;
            for (int t = 0; t < kc; ++t) {
                const float b = (lo + t < P.nb) ? sp->boundaries[lo + t] : INFINITY;
                c += (z[i] > b) ? 1 : 0;
            }
        } else {
            for (int t = 0; t < P.nb; ++t) c += (z[i] > sp->boundaries[t]) ? 1 : 0;
        }
        idx[i] = static_cast<uint8_t>(c & 0xFF);
    }
    return TQ_OK;
}

// ---- device-pointer entry points -------------------------------------------

tq_status tq_encode_batch_device(const tq_space *sp, const float *X, size_t n, uint8_t *out,
                                 void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(X, n * sp->dim * 4, "X")) != TQ_OK) return st;
    if ((st = check_dev(out, n * sp->code_size, "out")) != TQ_OK) return st;
    TQ_CUDA(tq::launch_encode(sp->P, sp->T, X, n, out, (cudaStream_t)stream), "encode kernel");
    return TQ_OK;
}

tq_status tq_prepare_queries_device(const tq_space *sp, const float *Q, size_t m, float *q_rot,
                                    float *s_q, float *norms, void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (m == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(Q, m * sp->dim * 4, "queries")) != TQ_OK) return st;
    if ((st = check_dev(q_rot, m * sp->D * 4, "q_rot")) != TQ_OK) return st;
    if ((st = check_dev(s_q, m * sp->D * 4, "s_q")) != TQ_OK) return st;
    if ((st = check_dev(norms, m * 8, "norms")) != TQ_OK) return st;
    TQ_CUDA(tq::launch_prepare(sp->P, sp->T, Q, m, q_rot, s_q, norms, (cudaStream_t)stream),
            "prepare kernel");
    return TQ_OK;
}

tq_status tq_prepare_query(const tq_space *csp, const float *query, float *q_rot, float *s_q,
                           float *norms) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (!query || !q_rot || !s_q || !norms) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    cudaStream_t s = sp->host_stream[0];
    const size_t D = sp->D, dim = sp->dim;
    Scratch buf;
    TQ_CUDA(buf.alloc(sizeof(float) * (dim + 2 * D + 2), s), "cudaMallocAsync(prepare)");
    float *dq = static_cast<float *>(buf.p), *dr = dq + dim, *ds = dr + D, *dn = ds + D;
    TQ_CUDA(cudaMemcpyAsync(dq, query, dim * 4, cudaMemcpyHostToDevice, s), "H2D query");
    TQ_CUDA(tq::launch_prepare(sp->P, sp->T, dq, 1, dr, ds, dn, s), "prepare kernel");
    TQ_CUDA(cudaMemcpyAsync(q_rot, dr, D * 4, cudaMemcpyDeviceToHost, s), "D2H q_rot");
    TQ_CUDA(cudaMemcpyAsync(s_q, ds, D * 4, cudaMemcpyDeviceToHost, s), "D2H s_q");
    TQ_CUDA(cudaMemcpyAsync(norms, dn, 8, cudaMemcpyDeviceToHost, s), "D2H norms");
    TQ_CUDA(cudaStreamSynchronize(s), "prepare_query");
    return TQ_OK;
}

}  // extern "C"

namespace {

// The 1->N scan launch of every distance_1_to_n entry point; while the space's
// scan timer is on, it is bracketed by a pair of CUDA events on its stream.
cudaError_t scan_1_to_n(const tq_space *csp, const float *q_rot, const float *s_q,
                        const float *norms, const uint8_t *codes, size_t n, float *out,
                        cudaStream_t s) {
    auto *sp = const_cast<tq_space *>(csp);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    {
        std::lock_guard<std::mutex> lk(sp->timer_mu);
        if (sp->timer_on) {
            while (sp->timer_events.size() < 2 * (sp->timer_used + 1)) {
                cudaEvent_t e = nullptr;
                const cudaError_t r = cudaEventCreate(&e);
                if (r != cudaSuccess) return r;
                sp->timer_events.push_back(e);
            }
            ev[0] = sp->timer_events[2 * sp->timer_used];
            ev[1] = sp->timer_events[2 * sp->timer_used + 1];
            ++sp->timer_used;
        }
    }
    cudaError_t e = ev[0] ? cudaEventRecord(ev[0], s) : cudaSuccess;
    if (e == cudaSuccess) e = tq::launch_scan_1_to_n(sp->P, sp->T, q_rot, s_q, norms, codes, n, out, s);
    if (e == cudaSuccess && ev[1]) e = cudaEventRecord(ev[1], s);
    return e;
}

}  // namespace

extern "C" {

tq_status tq_space_scan_timer(tq_space *sp, int enable) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    std::lock_guard<std::mutex> lk(sp->timer_mu);
    sp->timer_on = enable != 0;
    if (enable) sp->timer_used = 0;
    return TQ_OK;
}

tq_status tq_space_scan_timer_read(tq_space *sp, double *total_ms, uint64_t *launches) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    DeviceGuard g(sp->device);
    std::lock_guard<std::mutex> lk(sp->timer_mu);
    double total = 0.0;
    for (size_t i = 0; i < sp->timer_used; ++i) {
        TQ_CUDA(cudaEventSynchronize(sp->timer_events[2 * i + 1]), "scan timer sync");
        float ms = 0.0f;
        TQ_CUDA(cudaEventElapsedTime(&ms, sp->timer_events[2 * i], sp->timer_events[2 * i + 1]),
                "scan timer");
        total += ms;
    }
    if (total_ms) *total_ms = total;
    if (launches) *launches = sp->timer_used;
    return TQ_OK;
}

tq_status tq_distance_1_to_n_device(const tq_space *sp, const float *query,
                                    const uint8_t *codes, size_t n, float *out, void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(query, sp->dim * 4, "query")) != TQ_OK) return st;
    if ((st = check_dev(codes, n * sp->code_size, "codes")) != TQ_OK) return st;
    if ((st = check_codes_align(codes, "codes")) != TQ_OK) return st;
    if ((st = check_dev(out, n * 4, "out")) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    Scratch scr;
    TQ_CUDA(scr.alloc(sizeof(float) * (2 * sp->D + 2), s), "cudaMallocAsync(prepared query)");
    float *q_rot = static_cast<float *>(scr.p), *s_q = q_rot + sp->D, *norms = s_q + sp->D;
    TQ_CUDA(tq::launch_prepare(sp->P, sp->T, query, 1, q_rot, s_q, norms, s), "prepare kernel");
    TQ_CUDA(scan_1_to_n(sp, q_rot, s_q, norms, codes, n, out, s), "scan kernel");
    return TQ_OK;
}

tq_status tq_space_take_device_status(const tq_space *sp, int *code) {
    if (code) *code = 0;
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    DeviceGuard g(sp->device);
    return take_status(sp, code);
}

tq_status tq_distance_1_to_n_prepared_device(const tq_space *sp, const float *q_rot,
                                             const float *s_q, const float *norms,
                                             const uint8_t *codes, size_t n, float *out,
                                             void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(q_rot, sp->D * 4, "q_rot")) != TQ_OK) return st;
    if ((st = check_dev(s_q, sp->D * 4, "s_q")) != TQ_OK) return st;
    if ((st = check_dev(norms, 8, "norms")) != TQ_OK) return st;
    if ((st = check_dev(codes, n * sp->code_size, "codes")) != TQ_OK) return st;
    if ((st = check_codes_align(codes, "codes")) != TQ_OK) return st;
    if ((st = check_dev(out, n * 4, "out")) != TQ_OK) return st;
    TQ_CUDA(scan_1_to_n(sp, q_rot, s_q, norms, codes, n, out, (cudaStream_t)stream), "scan kernel");
    return TQ_OK;
}

}  // extern "C"

namespace {

// Fixed device scratch of tq_distance_1_to_n_device_noalloc: the prepared
// query (q_rot, s_q, |q|^2, |q|) of the largest supported padded dim.
constexpr size_t kNoAllocScratchFloats = 2 * (size_t(1) << tq::kMaxLogD) + 2;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocSlot {
    std::once_flag once;
    float *ptr = nullptr;
    cudaError_t err = cudaSuccess;
};
NoAllocSlot g_noalloc_slots[kNoAllocMaxDevices];

// Device address of this device's copy of the array (looked up once per
// device, with that device current; the host-side name is not a device
// address).
tq_status noalloc_scratch(int device, float **out) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        return fail(TQ_ERR_NOT_SUPPORTED, "device %d: no static scratch slot", device);
    NoAllocSlot &slot = g_noalloc_slots[device];
    std::call_once(slot.once, [&] {
        void *p = nullptr;
        slot.err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (slot.err == cudaSuccess) slot.ptr = static_cast<float *>(p);
    });
    if (slot.err != cudaSuccess) return cuda_fail(slot.err, "cudaGetSymbolAddress(static scratch)");
    *out = slot.ptr;
    return TQ_OK;
}

}  // namespace

extern "C" {

tq_status tq_distance_1_to_n_device_noalloc(const tq_space *sp, const float *query,
                                            const uint8_t *codes, size_t n, float *out,
                                            void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    const size_t need = 2 * sp->D + 2;
    if (need > kNoAllocScratchFloats)
        return fail(TQ_ERR_INVALID_ARGUMENT,
                    "distance_1_to_n_device_noalloc: padded dim %zu needs %zu floats of scratch, "
                    "the static scratch holds %zu",
                    sp->D, need, kNoAllocScratchFloats);
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(query, sp->dim * 4, "query")) != TQ_OK) return st;
    if ((st = check_dev(codes, n * sp->code_size, "codes")) != TQ_OK) return st;
    if ((st = check_codes_align(codes, "codes")) != TQ_OK) return st;
    if ((st = check_dev(out, n * 4, "out")) != TQ_OK) return st;
    float *scratch = nullptr;
    if ((st = noalloc_scratch(sp->device, &scratch)) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    float *q_rot = scratch, *s_q = scratch + sp->D, *norms = scratch + 2 * sp->D;
    TQ_CUDA(tq::launch_prepare(sp->P, sp->T, query, 1, q_rot, s_q, norms, s), "prepare kernel");
    TQ_CUDA(tq::launch_scan_1_to_n(sp->P, sp->T, q_rot, s_q, norms, codes, n, out, s), "scan kernel");
    return TQ_OK;
}

tq_status tq_distance_m_to_n_device(const tq_space *sp, const float *queries, size_t m,
                                    const uint8_t *codes, size_t n, float *out,
                                    tq_precision precision, void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if ((st = mton_precision_ok(precision, false)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(queries, m * sp->dim * 4, "queries")) != TQ_OK) return st;
    if ((st = check_dev(codes, n * sp->code_size, "codes")) != TQ_OK) return st;
    if ((st = check_codes_align(codes, "codes")) != TQ_OK) return st;
    if ((st = check_dev(out, m * n * 4, "out")) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t mchunk = MtonRunner::row_chunk(sp, false, precision);
    for (size_t m0 = 0; m0 < m; m0 += mchunk) {
        const size_t mc = std::min(mchunk, m - m0);
        MtonRunner r(const_cast<tq_space *>(sp), false, precision, mc);
        if ((st = r.prepare_rows(queries + m0 * sp->dim, s)) != TQ_OK) return st;
        if ((st = r.run_cols(codes, n, out + m0 * n, n, s)) != TQ_OK) return st;
        if ((st = r.finish(s)) != TQ_OK) return st;
    }
    return TQ_OK;
}

tq_status tq_distance_m_to_n_symmetric_device(const tq_space *sp, const uint8_t *A, size_t m,
                                              const uint8_t *B, size_t n, float *out,
                                              tq_precision precision, void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if ((st = mton_precision_ok(precision, true)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(A, m * sp->code_size, "codes_a")) != TQ_OK) return st;
    if ((st = check_dev(B, n * sp->code_size, "codes_b")) != TQ_OK) return st;
    if ((st = check_codes_align(A, "codes_a")) != TQ_OK) return st;
    if ((st = check_codes_align(B, "codes_b")) != TQ_OK) return st;
    if ((st = check_dev(out, m * n * 4, "out")) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t mchunk = MtonRunner::row_chunk(sp, true, precision);
    for (size_t m0 = 0; m0 < m; m0 += mchunk) {
        const size_t mc = std::min(mchunk, m - m0);
        MtonRunner r(const_cast<tq_space *>(sp), true, precision, mc);
        if ((st = r.prepare_rows(A + m0 * sp->code_size, s)) != TQ_OK) return st;
        if ((st = r.run_cols(B, n, out + m0 * n, n, s)) != TQ_OK) return st;
        if ((st = r.finish(s)) != TQ_OK) return st;
    }
    return TQ_OK;
}

// ---- host-pointer entry points ---------------------------------------------
// Inputs are streamed through the GPU in chunks of ~256 MB on two streams that
// alternate, so the copies of one chunk overlap the kernels of the other.

tq_status tq_encode_batch(const tq_space *csp, const float *X, size_t n, uint8_t *out) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    if (!X || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    const size_t row_bytes = sp->dim * 4;
    size_t rows = std::max<size_t>(4, (kChunkBytes / row_bytes) & ~size_t(3));
    rows = std::min(rows, n);
    Scratch buf[2];
    for (int k = 0; k < 2; ++k)
        TQ_CUDA(buf[k].alloc(rows * (row_bytes + sp->code_size), sp->host_stream[k]),
                "cudaMallocAsync(encode staging)");
    size_t chunk = 0;
    for (size_t r0 = 0; r0 < n; r0 += rows, ++chunk) {
        const size_t nr = std::min(rows, n - r0);
        cudaStream_t s = sp->host_stream[chunk & 1];
        float *dX = static_cast<float *>(buf[chunk & 1].p);
        uint8_t *dC = reinterpret_cast<uint8_t *>(dX) + rows * row_bytes;
        TQ_CUDA(cudaMemcpyAsync(dX, X + r0 * sp->dim, nr * row_bytes, cudaMemcpyHostToDevice, s),
                "H2D X");
        TQ_CUDA(tq::launch_encode(sp->P, sp->T, dX, nr, dC, s), "encode kernel");
        TQ_CUDA(cudaMemcpyAsync(out + r0 * sp->code_size, dC, nr * sp->code_size,
                                cudaMemcpyDeviceToHost, s),
                "D2H codes");
    }
    for (auto &s : sp->host_stream) TQ_CUDA(cudaStreamSynchronize(s), "encode");
    return TQ_OK;
}

tq_status tq_distance_1_to_n(const tq_space *csp, const float *query, const uint8_t *codes,
                             size_t n, float *out) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    if (!query || !codes || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    const size_t cs = sp->code_size;
    size_t per = std::max<size_t>(1, kChunkBytes / cs);
    per = std::min(per, n);
    cudaStream_t s0 = sp->host_stream[0];
    Scratch qs;
    TQ_CUDA(qs.alloc(sizeof(float) * (sp->dim + 2 * sp->D + 2), s0), "cudaMallocAsync(query)");
    float *dq = static_cast<float *>(qs.p), *q_rot = dq + sp->dim, *s_q = q_rot + sp->D,
          *norms = s_q + sp->D;
    TQ_CUDA(cudaMemcpyAsync(dq, query, sp->dim * 4, cudaMemcpyHostToDevice, s0), "H2D query");
    TQ_CUDA(tq::launch_prepare(sp->P, sp->T, dq, 1, q_rot, s_q, norms, s0), "prepare kernel");
    cudaEvent_t ready;
    TQ_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
    cudaEventRecord(ready, s0);
    cudaStreamWaitEvent(sp->host_stream[1], ready, 0);
    Scratch buf[2];
    tq_status result = TQ_OK;
    for (int k = 0; k < 2 && result == TQ_OK; ++k) {
        cudaError_t e = buf[k].alloc(per * (cs + 4) + 16, sp->host_stream[k]);
        if (e != cudaSuccess) result = cuda_fail(e, "cudaMallocAsync(scan staging)");
    }
    size_t chunk = 0;
    for (size_t c0 = 0; c0 < n && result == TQ_OK; c0 += per, ++chunk) {
        const size_t nc = std::min(per, n - c0);
        cudaStream_t s = sp->host_stream[chunk & 1];
        uint8_t *dC = static_cast<uint8_t *>(buf[chunk & 1].p);
        float *dO = reinterpret_cast<float *>(dC + ((per * cs + 15) & ~size_t(15)));
        cudaError_t e = cudaMemcpyAsync(dC, codes + c0 * cs, nc * cs, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = tq::launch_scan_1_to_n(sp->P, sp->T, q_rot, s_q, norms, dC, nc, dO, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out + c0, dO, nc * 4, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) result = cuda_fail(e, "distance_1_to_n chunk");
    }
    for (auto &s : sp->host_stream) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess && result == TQ_OK) result = cuda_fail(e, "distance_1_to_n");
    }
    cudaEventDestroy(ready);
    if (result == TQ_OK) result = take_status(sp, nullptr);
    return result;
}

}  // extern "C"

namespace {

// Shared driver of the two host-pointer M x N entry points: the row side is
// uploaded and prepared once; the column side (codes) is streamed in chunks.
// Three streams: uploads (host_stream[1]), contractions (host_stream[0]) and
// downloads (a third stream), so that the H2D of chunk k+1, the kernels of
// chunk k and the pitched D2H of chunk k-1 overlap on separate engines.
tq_status mton_host(tq_space *sp, bool sym, tq_precision prec, const void *rows_host, size_t m,
                    const uint8_t *codes, size_t n, float *out) {
    const size_t cs = sp->code_size;
    const size_t row_bytes = sym ? m * cs : m * sp->dim * 4;
    size_t per = std::max<size_t>(1, std::min(kChunkBytes / cs, (kChunkBytes * 2) / (4 * m)));
    per = std::min(per, n);
    cudaStream_t sc = sp->host_stream[0], su = sp->host_stream[1];
    cudaStream_t sd = nullptr;
    TQ_CUDA(cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking), "cudaStreamCreate");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sguard{sd};
    Scratch rows;
    TQ_CUDA(rows.alloc(row_bytes, sc), "cudaMallocAsync(rows)");
    TQ_CUDA(cudaMemcpyAsync(rows.p, rows_host, row_bytes, cudaMemcpyHostToDevice, sc), "H2D rows");
    MtonRunner runner(sp, sym, prec, m);
    tq_status st = runner.prepare_rows(rows.p, sc);
    if (st != TQ_OK) return st;
    const size_t cbytes = (per * cs + 15) & ~size_t(15);
    Scratch buf[2];
    for (int k = 0; k < 2; ++k)
        TQ_CUDA(buf[k].alloc(cbytes + per * m * 4, sc), "cudaMallocAsync(m_to_n staging)");
    cudaEvent_t uploaded[2], computed[2], downloaded[2];
    for (int k = 0; k < 2; ++k) {
        TQ_CUDA(cudaEventCreateWithFlags(&uploaded[k], cudaEventDisableTiming), "event");
        TQ_CUDA(cudaEventCreateWithFlags(&computed[k], cudaEventDisableTiming), "event");
        TQ_CUDA(cudaEventCreateWithFlags(&downloaded[k], cudaEventDisableTiming), "event");
        // the staging buffers were allocated on sc: the other streams start after it
        cudaEventRecord(downloaded[k], sc);
        cudaEventRecord(computed[k], sc);
    }
    tq_status result = TQ_OK;
    size_t chunk = 0;
    for (size_t c0 = 0; c0 < n && result == TQ_OK; c0 += per, ++chunk) {
        const size_t nc = std::min(per, n - c0);
        const int k = (int)(chunk & 1);
        uint8_t *dC = static_cast<uint8_t *>(buf[k].p);
        float *dO = reinterpret_cast<float *>(dC + cbytes);
        // upload into buffer k once the contraction that last read it is done
        cudaError_t e = cudaStreamWaitEvent(su, computed[k], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dC, codes + c0 * cs, nc * cs, cudaMemcpyHostToDevice, su);
        if (e == cudaSuccess) e = cudaEventRecord(uploaded[k], su);
        // contract once uploaded and once the previous download of dO is done
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, uploaded[k], 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, downloaded[k], 0);
        if (e != cudaSuccess) { result = cuda_fail(e, "m_to_n upload"); break; }
        st = runner.run_cols(dC, nc, dO, nc, sc);
        if (st != TQ_OK) { result = st; break; }
        e = cudaEventRecord(computed[k], sc);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sd, computed[k], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(out + c0, n * 4, dO, nc * 4, nc * 4, m, cudaMemcpyDeviceToHost, sd);
        if (e == cudaSuccess) e = cudaEventRecord(downloaded[k], sd);
        if (e != cudaSuccess) result = cuda_fail(e, "m_to_n chunk");
    }
    for (cudaStream_t s : {su, sc, sd}) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess && result == TQ_OK) result = cuda_fail(e, "m_to_n");
    }
    if (result == TQ_OK) result = runner.finish(sc);
    for (int k = 0; k < 2; ++k) {
        cudaEventDestroy(uploaded[k]);
        cudaEventDestroy(computed[k]);
        cudaEventDestroy(downloaded[k]);
    }
    return result;
}

}  // namespace

extern "C" {

tq_status tq_distance_m_to_n(const tq_space *csp, const float *queries, size_t m,
                             const uint8_t *codes, size_t n, float *out, tq_precision precision) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if ((st = mton_precision_ok(precision, false)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    if (!queries || !codes || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    return mton_host(sp, false, precision, queries, m, codes, n, out);
}

tq_status tq_distance_m_to_n_symmetric(const tq_space *csp, const uint8_t *codes_a, size_t m,
                                       const uint8_t *codes_b, size_t n, float *out,
                                       tq_precision precision) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if ((st = mton_precision_ok(precision, true)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    if (!codes_a || !codes_b || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    return mton_host(sp, true, precision, codes_a, m, codes_b, n, out);
}

}  // extern "C"

// ---- rotated coordinates and QJL-corrected symmetric distances -------------
namespace {

constexpr size_t kSymqChunkBytes = size_t(512) << 20;     // FP32 column planes per chunk
constexpr size_t kSymqTcChunkBytes = size_t(2048) << 20;  // TF32 pairs: fewer, longer launches

size_t sq_round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Row planes built once (from row codes, or from a prepared code), column
// planes built per chunk; one two-accumulator contraction per chunk: the FP32
// CUDA-core kernel, or (split-TF32) the FP32 planes split into hi/lo TF32
// planes (K padded to 32, rows to 128 / 256) for the tcgen05 kernel.  Padded
// dims below 64 keep the FP32 kernel: a tile of so short a reduction is
// mostly padding.
struct SymqRunner {
    const tq_space *sp;
    int mode, ldk1, ldk2;
    bool tc;
    int K1p = 0, K2p = 0;
    size_t m = 0, m_pad = 0, per = 0;
    Scratch rows, cols, rows_bf, cols_bf;
    float *P1a = nullptr, *P2a = nullptr, *sa = nullptr;
    float *A1 = nullptr, *A2 = nullptr;  // hi then lo, m_pad x K1p / K2p each
    int *err = nullptr;

    SymqRunner(const tq_space *s, int md, bool split_tf32 = false)
        : sp(s), mode(md), tc(split_tf32 && s->D >= 64) {
        ldk1 = tq::symq_ldk((int)s->D);
        ldk2 = tq::symq_ldk(tq::symq_k2(md, (int)s->D));
        K1p = (int)sq_round_up((size_t)ldk1, 32);
        K2p = (int)sq_round_up((size_t)ldk2, 32);
    }
    size_t row_floats() const { return (size_t)ldk1 + ldk2 + 8; }
    tq_status alloc_rows(size_t rows_, cudaStream_t s) {
        m = rows_;
        TQ_CUDA(rows.alloc(sizeof(float) * row_floats() * m, s), "cudaMallocAsync(row planes)");
        P1a = static_cast<float *>(rows.p);
        P2a = P1a + m * ldk1;
        sa = P2a + m * ldk2;
        return TQ_OK;
    }
    tq_status prepare_rows(const uint8_t *A, size_t rows_, cudaStream_t s) {
        if (tc) return prepare_rows_tc(A, rows_, s);
        tq_status st = alloc_rows(rows_, s);
        if (st != TQ_OK) return st;
        TQ_CUDA(tq::launch_symq_planes(sp->P, sp->T, A, m, mode, true, P1a, ldk1, P2a, ldk2, sa, s),
                "symmetric planes kernel");
        return TQ_OK;
    }
    // The row planes straight into hi/lo TF32 pairs (m_pad x K1p, m_pad x
    // K2p); the light variant's sign plane is exact and has no lo plane.
    tq_status prepare_rows_tc(const uint8_t *A, size_t rows_, cudaStream_t s) {
        m = rows_;
        TQ_CUDA(rows.alloc(sizeof(float) * 8 * m, s), "cudaMallocAsync(row scalars)");
        sa = static_cast<float *>(rows.p);
        m_pad = sq_round_up(m, 128);
        const size_t e1 = m_pad * K1p, e2 = m_pad * K2p;  // floats per plane
        TQ_CUDA(rows_bf.alloc(sizeof(float) * 2 * (e1 + e2), s), "cudaMallocAsync(row TF32 planes)");
        A1 = static_cast<float *>(rows_bf.p);
        A2 = A1 + 2 * e1;
        TQ_CUDA(tq::launch_symq_planes_tf32(sp->P, sp->T, A, m, m_pad, mode, true, A1, A1 + e1, K1p, A2,
                                            light() ? nullptr : A2 + e2, K2p, sa, s),
                "symmetric TF32 planes kernel");
        return TQ_OK;
    }
    bool light() const { return mode == tq::SYMQ_LIGHT; }
    tq_status prepare_row_from_prepared(const float *recon, const float *sign, const float *sc,
                                        cudaStream_t s) {
        tq_status st = alloc_rows(1, s);
        if (st != TQ_OK) return st;
        TQ_CUDA(tq::launch_symq_prepared_row(recon, sign, sc, (int)sp->D, P1a, ldk1, P2a, ldk2, sa, s),
                "prepared row kernel");
        return TQ_OK;
    }
    // out[:, 0:n] (leading dimension ldo) for n column codes
    tq_status run_cols(const uint8_t *B, size_t n, float *out, size_t ldo, cudaStream_t s) {
        if (tc) return run_cols_tc(B, n, out, ldo, s);
        if (!per) {
            per = std::max<size_t>(64, kSymqChunkBytes / (sizeof(float) * row_floats()));
            per = std::min(per, std::max<size_t>(n, 1));
            TQ_CUDA(cols.alloc(sizeof(float) * row_floats() * per, s), "cudaMallocAsync(column planes)");
        }
        float *P1b = static_cast<float *>(cols.p), *P2b = P1b + per * ldk1, *sb = P2b + per * ldk2;
        for (size_t c0 = 0; c0 < n; c0 += per) {
            const size_t nc = std::min(per, n - c0);
            TQ_CUDA(tq::launch_symq_planes(sp->P, sp->T, B + c0 * sp->code_size, nc, mode, false, P1b,
                                           ldk1, P2b, ldk2, sb, s),
                    "symmetric planes kernel");
            TQ_CUDA(tq::launch_symq_gemm(P1a, P2a, sa, m, P1b, P2b, sb, nc, ldk1, ldk2, out + c0, ldo, s),
                    "symmetric contraction kernel");
        }
        return TQ_OK;
    }
    tq_status run_cols_tc(const uint8_t *B, size_t n, float *out, size_t ldo, cudaStream_t s) {
        const size_t bf_row = (size_t)8 * (K1p + K2p);  // hi + lo floats of both planes
        if (!per) {
            per = std::max<size_t>(256, (kSymqTcChunkBytes / (bf_row + 32)) & ~size_t(255));
            per = std::min(per, sq_round_up(n, 256));
            TQ_CUDA(cols.alloc(sizeof(float) * 8 * per, s), "cudaMallocAsync(column scalars)");
            TQ_CUDA(cols_bf.alloc(bf_row * per + 16, s), "cudaMallocAsync(column TF32 planes)");
            err = reinterpret_cast<int *>(static_cast<unsigned char *>(cols_bf.p) + bf_row * per);
            TQ_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s), "memset");
        }
        float *sb = static_cast<float *>(cols.p);
        const size_t b1 = per * K1p, b2 = per * K2p;  // floats per plane
        float *B1 = static_cast<float *>(cols_bf.p), *B2 = B1 + 2 * b1;
        const size_t a1 = m_pad * K1p, a2 = m_pad * K2p;
        for (size_t c0 = 0; c0 < n; c0 += per) {
            const size_t nc = std::min(per, n - c0), nc_pad = sq_round_up(nc, 256);
            TQ_CUDA(tq::launch_symq_planes_tf32(sp->P, sp->T, B + c0 * sp->code_size, nc, nc_pad, mode,
                                                false, B1, B1 + b1, K1p, B2, light() ? nullptr : B2 + b2,
                                                K2p, sb, s),
                    "symmetric TF32 planes kernel");
            TQ_CUDA(tq::launch_tc_symq(A1, A1 + a1, B1, B1 + b1, K1p, A2, A2 + a2, B2, B2 + b2, K2p,
                                       light(), m, m_pad, nc, nc_pad, sa, sb, out + c0, ldo, err, s),
                    "tcgen05 symmetric contraction kernel");
        }
        return TQ_OK;
    }
    // Reports a bounded wait that gave up inside the tensor-core kernel.
    tq_status finish(cudaStream_t s) {
        if (!err) return TQ_OK;
        int h = 0;
        TQ_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H status");
        TQ_CUDA(cudaStreamSynchronize(s), "sync");
        if (h != 0) return fail(TQ_ERR_TIMEOUT, "tensor-core kernel: a pipeline wait timed out (code %d)", h);
        return TQ_OK;
    }
};

// The QJL-corrected symmetric contractions run in FP32 (CUDA cores) or
// split-TF32 (tensor cores).  A BF16 pair is refused: its planes' rounding
// errors do not average out (see tc_symq_kernel) and exceed 1e-5.
tq_status symq_precision_ok(tq_precision p) {
    if (p == TQ_PRECISION_FP32 || p == TQ_PRECISION_SPLIT_TF32) return TQ_OK;
    if (p == TQ_PRECISION_SPLIT_BF16 || p == TQ_PRECISION_REFERENCE)
        return fail(TQ_ERR_NOT_SUPPORTED,
                    "QJL-corrected symmetric distances take TQ_PRECISION_FP32 or "
                    "TQ_PRECISION_SPLIT_TF32 (a BF16 pair is not accurate enough here)");
    return fail(TQ_ERR_INVALID_ARGUMENT, "unknown precision %d", (int)p);
}

int sym_mode(tq_sym_variant v) {
    switch (v) {
        case TQ_SYM_LIGHT: return tq::SYMQ_LIGHT;
        case TQ_SYM_FULL: return tq::SYMQ_FULL;
        case TQ_SYM_FULL_PREPARED: return tq::SYMQ_FULL_PREPARED;
        default: return -1;
    }
}

}  // namespace

extern "C" {

tq_status tq_rotated_coords_batch_device(const tq_space *sp, const float *X, size_t n, float *out,
                                         void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(X, n * sp->dim * 4, "X")) != TQ_OK) return st;
    if ((st = check_dev(out, n * sp->D * 4, "out")) != TQ_OK) return st;
    TQ_CUDA(tq::launch_rotated_coords(sp->P, sp->T, X, n, out, (cudaStream_t)stream),
            "rotated coordinates kernel");
    return TQ_OK;
}

tq_status tq_rotated_coords_batch(const tq_space *csp, const float *X, size_t n, float *out) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    if (!X || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    cudaStream_t s = sp->host_stream[0];
    const size_t in_row = sp->dim * 4, out_row = sp->D * 4;
    const size_t rows = std::min(n, std::max<size_t>(1, kChunkBytes / (in_row + out_row)));
    Scratch buf;
    TQ_CUDA(buf.alloc(rows * (in_row + out_row), s), "cudaMallocAsync(rotated staging)");
    float *dX = static_cast<float *>(buf.p);
    float *dO = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(dX) + rows * in_row);
    for (size_t r0 = 0; r0 < n; r0 += rows) {
        const size_t nr = std::min(rows, n - r0);
        TQ_CUDA(cudaMemcpyAsync(dX, X + r0 * sp->dim, nr * in_row, cudaMemcpyHostToDevice, s), "H2D X");
        TQ_CUDA(tq::launch_rotated_coords(sp->P, sp->T, dX, nr, dO, s), "rotated coordinates kernel");
        TQ_CUDA(cudaMemcpyAsync(out + r0 * sp->D, dO, nr * out_row, cudaMemcpyDeviceToHost, s), "D2H");
    }
    TQ_CUDA(cudaStreamSynchronize(s), "rotated_coords_batch");
    return TQ_OK;
}

tq_status tq_distance_m_to_n_symmetric_qjl_device(const tq_space *sp, const uint8_t *A, size_t m,
                                                  const uint8_t *B, size_t n, float *out,
                                                  tq_sym_variant variant, tq_precision precision,
                                                  void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    const int mode = sym_mode(variant);
    if (mode < 0) return fail(TQ_ERR_INVALID_ARGUMENT, "unknown symmetric variant %d", (int)variant);
    if ((st = symq_precision_ok(precision)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(A, m * sp->code_size, "codes_a")) != TQ_OK) return st;
    if ((st = check_dev(B, n * sp->code_size, "codes_b")) != TQ_OK) return st;
    if ((st = check_dev(out, m * n * 4, "out")) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    SymqRunner r(sp, mode, precision == TQ_PRECISION_SPLIT_TF32);
    if ((st = r.prepare_rows(A, m, s)) != TQ_OK) return st;
    if ((st = r.run_cols(B, n, out, n, s)) != TQ_OK) return st;
    return r.finish(s);
}

tq_status tq_distance_m_to_n_symmetric_qjl(const tq_space *csp, const uint8_t *codes_a, size_t m,
                                           const uint8_t *codes_b, size_t n, float *out,
                                           tq_sym_variant variant, tq_precision precision) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    const int mode = sym_mode(variant);
    if (mode < 0) return fail(TQ_ERR_INVALID_ARGUMENT, "unknown symmetric variant %d", (int)variant);
    if ((st = symq_precision_ok(precision)) != TQ_OK) return st;
    if (m == 0 || n == 0) return TQ_OK;
    if (!codes_a || !codes_b || !out) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    cudaStream_t s = sp->host_stream[0];
    const size_t cs = sp->code_size;
    Scratch dA;
    TQ_CUDA(dA.alloc(m * cs, s), "cudaMallocAsync(codes_a)");
    TQ_CUDA(cudaMemcpyAsync(dA.p, codes_a, m * cs, cudaMemcpyHostToDevice, s), "H2D codes_a");
    SymqRunner r(sp, mode, precision == TQ_PRECISION_SPLIT_TF32);
    if ((st = r.prepare_rows(static_cast<uint8_t *>(dA.p), m, s)) != TQ_OK) return st;
    size_t per = std::max<size_t>(1, std::min(kChunkBytes / cs, (kChunkBytes * 2) / (4 * m)));
    per = std::min(per, n);
    Scratch buf;
    const size_t cbytes = (per * cs + 15) & ~size_t(15);
    TQ_CUDA(buf.alloc(cbytes + per * m * 4, s), "cudaMallocAsync(symmetric staging)");
    uint8_t *dB = static_cast<uint8_t *>(buf.p);
    float *dO = reinterpret_cast<float *>(dB + cbytes);
    for (size_t c0 = 0; c0 < n; c0 += per) {
        const size_t nc = std::min(per, n - c0);
        TQ_CUDA(cudaMemcpyAsync(dB, codes_b + c0 * cs, nc * cs, cudaMemcpyHostToDevice, s), "H2D codes_b");
        if ((st = r.run_cols(dB, nc, dO, nc, s)) != TQ_OK) return st;
        TQ_CUDA(cudaMemcpy2DAsync(out + c0, n * 4, dO, nc * 4, nc * 4, m, cudaMemcpyDeviceToHost, s),
                "D2H distances");
    }
    TQ_CUDA(cudaStreamSynchronize(s), "distance_m_to_n_symmetric (QJL)");
    return r.finish(s);
}

tq_status tq_prepare_symmetric_query(const tq_space *csp, const uint8_t *code, float *recon_q,
                                     float *sign_q, float *scalars) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (!code || !recon_q || !sign_q || !scalars) return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    cudaStream_t s = sp->host_stream[0];
    const int ldk1 = tq::symq_ldk((int)sp->D), ldk2 = tq::symq_ldk((int)sp->D);
    Scratch buf;
    const size_t cbytes = (sp->code_size + 15) & ~size_t(15);
    TQ_CUDA(buf.alloc(cbytes + sizeof(float) * (ldk1 + ldk2 + 8), s), "cudaMallocAsync(prepare)");
    uint8_t *dc = static_cast<uint8_t *>(buf.p);
    float *P1 = reinterpret_cast<float *>(dc + cbytes), *P2 = P1 + ldk1, *sc = P2 + ldk2;
    TQ_CUDA(cudaMemcpyAsync(dc, code, sp->code_size, cudaMemcpyHostToDevice, s), "H2D code");
    TQ_CUDA(tq::launch_symq_planes(sp->P, sp->T, dc, 1, tq::SYMQ_PREPARE, true, P1, ldk1, P2, ldk2,
                                   sc, s),
            "symmetric planes kernel");
    float sc8[8];
    TQ_CUDA(cudaMemcpyAsync(recon_q, P1, sp->D * 4, cudaMemcpyDeviceToHost, s), "D2H recon");
    TQ_CUDA(cudaMemcpyAsync(sign_q, P2, sp->D * 4, cudaMemcpyDeviceToHost, s), "D2H sign");
    TQ_CUDA(cudaMemcpyAsync(sc8, sc, sizeof(sc8), cudaMemcpyDeviceToHost, s), "D2H scalars");
    TQ_CUDA(cudaStreamSynchronize(s), "prepare_symmetric_query");
    scalars[0] = sc8[1];  // norm
    scalars[1] = sc8[3];  // gamma
    scalars[2] = sc8[4];  // sigma
    scalars[3] = sc8[5];  // scale * gamma
    scalars[4] = sc8[6];  // (pi / 2D) * gamma
    return TQ_OK;
}

tq_status tq_distance_1_to_n_symmetric_full_device(const tq_space *sp, const float *recon_q,
                                                   const float *sign_q, const float *scalars,
                                                   const uint8_t *codes, size_t n, float *out,
                                                   void *stream) {
    tq_status st = need_device(sp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    DeviceGuard g(sp->device);
    if ((st = check_dev(recon_q, sp->D * 4, "recon_q")) != TQ_OK) return st;
    if ((st = check_dev(sign_q, sp->D * 4, "sign_q")) != TQ_OK) return st;
    if ((st = check_dev(scalars, 5 * 4, "scalars")) != TQ_OK) return st;
    if ((st = check_dev(codes, n * sp->code_size, "codes")) != TQ_OK) return st;
    if ((st = check_dev(out, n * 4, "out")) != TQ_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    SymqRunner r(sp, tq::SYMQ_FULL_PREPARED);
    if ((st = r.prepare_row_from_prepared(recon_q, sign_q, scalars, s)) != TQ_OK) return st;
    return r.run_cols(codes, n, out, n, s);
}

tq_status tq_distance_1_to_n_symmetric_full(const tq_space *csp, const float *recon_q,
                                            const float *sign_q, const float *scalars,
                                            const uint8_t *codes, size_t n, float *out) {
    tq_status st = need_device(csp);
    if (st != TQ_OK) return st;
    if (n == 0) return TQ_OK;
    if (!recon_q || !sign_q || !scalars || !codes || !out)
        return fail(TQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    auto *sp = const_cast<tq_space *>(csp);
    std::lock_guard<std::mutex> lock(sp->host_mu);
    DeviceGuard g(sp->device);
    if ((st = ensure_host_streams(sp)) != TQ_OK) return st;
    cudaStream_t s = sp->host_stream[0];
    const size_t D = sp->D, cs = sp->code_size;
    Scratch q;
    TQ_CUDA(q.alloc(sizeof(float) * (2 * D + 8), s), "cudaMallocAsync(prepared code)");
    float *dr = static_cast<float *>(q.p), *ds = dr + D, *dsc = ds + D;
    TQ_CUDA(cudaMemcpyAsync(dr, recon_q, D * 4, cudaMemcpyHostToDevice, s), "H2D recon_q");
    TQ_CUDA(cudaMemcpyAsync(ds, sign_q, D * 4, cudaMemcpyHostToDevice, s), "H2D sign_q");
    TQ_CUDA(cudaMemcpyAsync(dsc, scalars, 5 * 4, cudaMemcpyHostToDevice, s), "H2D scalars");
    SymqRunner r(sp, tq::SYMQ_FULL_PREPARED);
    if ((st = r.prepare_row_from_prepared(dr, ds, dsc, s)) != TQ_OK) return st;
    const size_t per = std::min(n, std::max<size_t>(1, kChunkBytes / (cs + 4)));
    Scratch buf;
    const size_t cbytes = (per * cs + 15) & ~size_t(15);
    TQ_CUDA(buf.alloc(cbytes + per * 4, s), "cudaMallocAsync(symmetric staging)");
    uint8_t *dB = static_cast<uint8_t *>(buf.p);
    float *dO = reinterpret_cast<float *>(dB + cbytes);
    for (size_t c0 = 0; c0 < n; c0 += per) {
        const size_t nc = std::min(per, n - c0);
        TQ_CUDA(cudaMemcpyAsync(dB, codes + c0 * cs, nc * cs, cudaMemcpyHostToDevice, s), "H2D codes");
        if ((st = r.run_cols(dB, nc, dO, nc, s)) != TQ_OK) return st;
        TQ_CUDA(cudaMemcpyAsync(out + c0, dO, nc * 4, cudaMemcpyDeviceToHost, s), "D2H distances");
    }
    TQ_CUDA(cudaStreamSynchronize(s), "distance_1_to_n_symmetric_full");
    return TQ_OK;
}

}  // extern "C"
