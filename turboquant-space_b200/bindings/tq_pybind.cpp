// tq_pybind.cpp -- a pybind11 `_turboquant` extension over the C ABI
// (include/turboquant_b200.h): the module the reference's Python package
// imports (python/turboquant/__init__.py: `from ._turboquant import
// TurboQuantSpace`), with the classes, method names, keyword names, defaults,
// return types and ValueError texts of its bindings (bindings.cpp:53-335), so
// that the reference's package and tests run unchanged on the GPU library.
//
// Every call goes through the C ABI with host pointers (synchronous, like the
// reference).  Errors of the C ABI raise ValueError (invalid arguments),
// MemoryError (out of memory) or RuntimeError (everything else).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "turboquant_b200.h"

namespace py = pybind11;

namespace {

void check(tq_status st) {
    if (st == TQ_OK) return;
    const std::string msg = tq_last_error();
    if (st == TQ_ERR_INVALID_ARGUMENT) throw py::value_error(msg);
    if (st == TQ_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
    throw std::runtime_error(msg);
}

// A float32 input of `ndim` dims whose last extent is `last` (the reference's
// checks and texts, bindings.cpp:14-36: format, ndim, length or dim, last
// stride; the row stride is not checked there, so rows that are not packed
// are gathered here instead of read past).
struct FloatIn {
    const float *ptr = nullptr;
    size_t rows = 1;
    std::vector<float> gathered;
};

FloatIn float_in(const py::buffer &buf, size_t last, const char *name, int ndim) {
    const py::buffer_info info = buf.request();
    const std::string n(name);
    if (info.format != py::format_descriptor<float>::format())
        throw py::value_error(n + ": expected float32");
    if (info.ndim != ndim) throw py::value_error(n + ": wrong ndim");
    if (ndim == 1 && info.shape[0] != (py::ssize_t)last) throw py::value_error(n + ": wrong length");
    if (ndim == 2 && info.shape[1] != (py::ssize_t)last) throw py::value_error(n + ": wrong dim");
    if (info.strides[info.ndim - 1] != (py::ssize_t)sizeof(float))
        throw py::value_error(n + ": must be C-contiguous float32");
    FloatIn in;
    in.ptr = static_cast<const float *>(info.ptr);
    if (ndim == 2) {
        in.rows = (size_t)info.shape[0];
        const py::ssize_t row_stride = info.strides[0];
        if (in.rows > 1 && row_stride != (py::ssize_t)(last * sizeof(float))) {
            in.gathered.resize(in.rows * last);
            for (size_t r = 0; r < in.rows; ++r)
                std::memcpy(in.gathered.data() + r * last,
                            static_cast<const char *>(info.ptr) + (py::ssize_t)r * row_stride,
                            last * sizeof(float));
            in.ptr = in.gathered.data();
        }
    }
    return in;
}

// A uint8 buffer of exactly `bytes` bytes, any shape (bindings.cpp:38-49).
uint8_t *bytes_exact(const py::buffer &buf, size_t bytes, const char *name, bool writable) {
    const py::buffer_info info = buf.request(writable);
    const std::string n(name);
    if (info.itemsize != 1) throw py::value_error(n + ": must be uint8");
    if ((size_t)info.size != bytes) throw py::value_error(n + ": wrong byte size");
    return static_cast<uint8_t *>(info.ptr);
}

// A batch of codes: uint8, a whole number of codes, any shape
// (bindings.cpp:156-218).  Non-contiguous buffers are copied.
struct CodesIn {
    const uint8_t *ptr = nullptr;
    size_t n = 0;
    std::vector<uint8_t> copy;
};

CodesIn codes_in(const py::buffer &buf, size_t cs) {
    const py::buffer_info info = buf.request();
    if (info.itemsize != 1) throw py::value_error("codes must be uint8");
    if ((size_t)info.size % cs != 0)
        throw py::value_error("codes size not a multiple of code_size_bytes");
    CodesIn c;
    c.n = (size_t)info.size / cs;
    bool packed = true;
    py::ssize_t expect = 1;
    for (py::ssize_t d = info.ndim - 1; d >= 0; --d) {
        if (info.shape[d] != 1 && info.strides[d] != expect) packed = false;
        expect *= info.shape[d];
    }
    if (packed) {
        c.ptr = static_cast<const uint8_t *>(info.ptr);
    } else {
        py::array_t<uint8_t, py::array::c_style | py::array::forcecast> a(
            py::reinterpret_borrow<py::object>(buf));
        c.copy.assign(a.data(), a.data() + a.size());
        c.ptr = c.copy.data();
    }
    return c;
}

}  // namespace

namespace {

// prepareQuery's result (space_turbo_quant.h:138-144): q_rot, s_q, |q|^2, |q|.
struct PreparedQuery {
    std::vector<float> q_rot, s_q;
    float q_norm_sq = 0.0f, q_norm = 0.0f;
};

// prepareSymmetricQuery's result (:146-160): the code's QJL-rotated
// reconstruction, its +-1 signs and {norm, gamma, sigma, scale gamma, (pi/2D) gamma}.
struct PreparedSymCode {
    std::vector<float> recon_q, sign_q;
    float scalars[5] = {0, 0, 0, 0, 0};
};

class Space {
  public:
    Space(size_t dim, int bits, uint64_t rot_seed, uint64_t qjl_seed, int num_threads) {
        tq_space *sp = nullptr;
        check(tq_space_create(dim, bits, rot_seed, qjl_seed, num_threads, -1, &sp));
        sp_.reset(sp);
        check(tq_space_get_info(sp, &info_));
    }
    size_t dim() const { return info_.dim; }
    size_t padded_dim() const { return info_.padded_dim; }
    bool padded() const { return info_.padded != 0; }
    int num_threads() const { return info_.num_threads; }
    size_t code_size() const { return info_.code_size; }
    int bits() const { return info_.bits_per_coord; }

    py::array_t<uint8_t> encode(const py::buffer &x) const {
        const FloatIn in = float_in(x, dim(), "input", 1);
        py::array_t<uint8_t> out((py::ssize_t)code_size());
        check(tq_encode_batch(sp_.get(), in.ptr, 1, out.mutable_data()));
        return out;
    }
    void encode_into(const py::buffer &x, const py::buffer &out) const {
        const FloatIn in = float_in(x, dim(), "input", 1);
        uint8_t *o = bytes_exact(out, code_size(), "code", true);
        check(tq_encode_batch(sp_.get(), in.ptr, 1, o));
    }
    py::array_t<uint8_t> encode_batch(const py::buffer &X) const {
        const FloatIn in = float_in(X, dim(), "input", 2);
        py::array_t<uint8_t> out({(py::ssize_t)in.rows, (py::ssize_t)code_size()});
        if (in.rows) check(tq_encode_batch(sp_.get(), in.ptr, in.rows, out.mutable_data()));
        return out;
    }
    void encode_batch_into(const py::buffer &X, const py::buffer &out) const {
        const FloatIn in = float_in(X, dim(), "input", 2);
        uint8_t *o = bytes_exact(out, in.rows * code_size(), "codes", true);
        if (in.rows) check(tq_encode_batch(sp_.get(), in.ptr, in.rows, o));
    }
    py::array_t<float> rotated_coords_batch(const py::buffer &X) const {
        const FloatIn in = float_in(X, dim(), "input", 2);
        py::array_t<float> out({(py::ssize_t)in.rows, (py::ssize_t)padded_dim()});
        if (in.rows) check(tq_rotated_coords_batch(sp_.get(), in.ptr, in.rows, out.mutable_data()));
        return out;
    }
    float distance(const py::buffer &q, const py::buffer &code) const {
        const FloatIn in = float_in(q, dim(), "query", 1);
        const uint8_t *c = bytes_exact(code, code_size(), "code", false);
        float d = 0.0f;
        check(tq_distance_1_to_n(sp_.get(), in.ptr, c, 1, &d));
        return d;
    }
    float distance_symmetric(const py::buffer &a, const py::buffer &b) const {
        const uint8_t *ca = bytes_exact(a, code_size(), "code_a", false);
        const uint8_t *cb = bytes_exact(b, code_size(), "code_b", false);
        float d = 0.0f;
        check(tq_distance_m_to_n_symmetric(sp_.get(), ca, 1, cb, 1, &d, TQ_PRECISION_FP32));
        return d;
    }
    py::array_t<float> distance_1_to_n(const py::buffer &q, const py::buffer &codes) const {
        const FloatIn in = float_in(q, dim(), "query", 1);
        const CodesIn c = codes_in(codes, code_size());
        py::array_t<float> out((py::ssize_t)c.n);
        if (c.n) check(tq_distance_1_to_n(sp_.get(), in.ptr, c.ptr, c.n, out.mutable_data()));
        return out;
    }
    py::array_t<float> distance_m_to_n(const py::buffer &Q, const py::buffer &codes) const {
        const FloatIn in = float_in(Q, dim(), "queries", 2);
        const CodesIn c = codes_in(codes, code_size());
        py::array_t<float> out({(py::ssize_t)in.rows, (py::ssize_t)c.n});
        if (in.rows && c.n)
            check(tq_distance_m_to_n(sp_.get(), in.ptr, in.rows, c.ptr, c.n, out.mutable_data(),
                                     TQ_PRECISION_FP32));
        return out;
    }
    py::array_t<float> symmetric(const py::buffer &a, const py::buffer &b, int variant) const {
        const CodesIn ca = codes_in(a, code_size()), cb = codes_in(b, code_size());
        py::array_t<float> out({(py::ssize_t)ca.n, (py::ssize_t)cb.n});
        if (!ca.n || !cb.n) return out;
        if (variant < 0)
            check(tq_distance_m_to_n_symmetric(sp_.get(), ca.ptr, ca.n, cb.ptr, cb.n,
                                               out.mutable_data(), TQ_PRECISION_FP32));
        else
            check(tq_distance_m_to_n_symmetric_qjl(sp_.get(), ca.ptr, ca.n, cb.ptr, cb.n,
                                                   out.mutable_data(), (tq_sym_variant)variant,
                                                   TQ_PRECISION_FP32));
        return out;
    }
    PreparedQuery prepare_query(const py::buffer &q) const {
        const FloatIn in = float_in(q, dim(), "query", 1);
        PreparedQuery pq;
        pq.q_rot.resize(padded_dim());
        pq.s_q.resize(padded_dim());
        float norms[2];
        check(tq_prepare_query(sp_.get(), in.ptr, pq.q_rot.data(), pq.s_q.data(), norms));
        pq.q_norm_sq = norms[0];
        pq.q_norm = norms[1];
        return pq;
    }
    PreparedSymCode prepare_symmetric_query(const py::buffer &code) const {
        const uint8_t *c = bytes_exact(code, code_size(), "code", false);
        PreparedSymCode p;
        p.recon_q.resize(padded_dim());
        p.sign_q.resize(padded_dim());
        check(tq_prepare_symmetric_query(sp_.get(), c, p.recon_q.data(), p.sign_q.data(), p.scalars));
        return p;
    }
    py::array_t<float> distance_1_to_n_symmetric_full(const PreparedSymCode &p,
                                                      const py::buffer &codes) const {
        const CodesIn c = codes_in(codes, code_size());
        py::array_t<float> out((py::ssize_t)c.n);
        if (c.n)
            check(tq_distance_1_to_n_symmetric_full(sp_.get(), p.recon_q.data(), p.sign_q.data(),
                                                    p.scalars, c.ptr, c.n, out.mutable_data()));
        return out;
    }
    float distance_symmetric_full_prepared(const PreparedSymCode &p, const py::buffer &code_b) const {
        const uint8_t *c = bytes_exact(code_b, code_size(), "code_b", false);
        float d = 0.0f;
        check(tq_distance_1_to_n_symmetric_full(sp_.get(), p.recon_q.data(), p.sign_q.data(),
                                                p.scalars, c, 1, &d));
        return d;
    }

  private:
    struct Del {
        void operator()(tq_space *s) const { tq_space_destroy(s); }
    };
    std::unique_ptr<tq_space, Del> sp_;
    tq_space_info info_{};
};

}  // namespace

PYBIND11_MODULE(_turboquant, m) {
    m.doc() = "TurboQuant on B200: the reference's _turboquant module over libtqb200's C ABI";

    py::class_<PreparedQuery>(m, "PreparedQuery");
    py::class_<PreparedSymCode>(m, "PreparedSymCode");

    // Symmetric variants of tq_distance_m_to_n_symmetric_qjl (-1: plain distBuild).
    constexpr int kPlain = -1;

    py::class_<Space>(m, "TurboQuantSpace")
        .def(py::init<size_t, int, uint64_t, uint64_t, int>(), py::arg("dim"),
             py::arg("bits_per_coord") = 4, py::arg("rot_seed") = 42ULL,
             py::arg("qjl_seed") = 137ULL, py::arg("num_threads") = 0)
        .def("dim", &Space::dim)
        .def("padded_dim", &Space::padded_dim)
        .def("padded", &Space::padded)
        .def("num_threads", &Space::num_threads)
        .def("code_size_bytes", &Space::code_size)
        .def("bits_per_coord", &Space::bits)
        .def("encode", &Space::encode, py::arg("x"))
        .def("encode_into", &Space::encode_into, py::arg("x"), py::arg("out"))
        .def("encode_batch", &Space::encode_batch, py::arg("X"))
        .def("encode_batch_into", &Space::encode_batch_into, py::arg("X"), py::arg("out"))
        .def("rotated_coords_batch", &Space::rotated_coords_batch, py::arg("X"))
        .def("distance", &Space::distance, py::arg("query"), py::arg("code"))
        .def("distance_symmetric", &Space::distance_symmetric, py::arg("code_a"), py::arg("code_b"))
        .def("distance_1_to_n", &Space::distance_1_to_n, py::arg("query"), py::arg("codes"))
        .def("distance_m_to_n", &Space::distance_m_to_n, py::arg("queries"), py::arg("codes"))
        .def("distance_m_to_n_symmetric",
             [](const Space &s, const py::buffer &a, const py::buffer &b) {
                 return s.symmetric(a, b, kPlain);
             },
             py::arg("codes_a"), py::arg("codes_b"))
        .def("distance_m_to_n_symmetric_full",
             [](const Space &s, const py::buffer &a, const py::buffer &b) {
                 return s.symmetric(a, b, TQ_SYM_FULL);
             },
             py::arg("codes_a"), py::arg("codes_b"))
        .def("distance_m_to_n_symmetric_light",
             [](const Space &s, const py::buffer &a, const py::buffer &b) {
                 return s.symmetric(a, b, TQ_SYM_LIGHT);
             },
             py::arg("codes_a"), py::arg("codes_b"))
        .def("prepare_query", &Space::prepare_query, py::arg("query"))
        .def("prepare_symmetric_query", &Space::prepare_symmetric_query, py::arg("code"))
        .def("distance_symmetric_full_prepared", &Space::distance_symmetric_full_prepared,
             py::arg("pq"), py::arg("code_b"))
        .def("distance_1_to_n_symmetric_full", &Space::distance_1_to_n_symmetric_full, py::arg("pq"),
             py::arg("codes"))
        .def("distance_m_to_n_symmetric_full_prepared",
             [](const Space &s, const py::buffer &a, const py::buffer &b) {
                 return s.symmetric(a, b, TQ_SYM_FULL_PREPARED);
             },
             py::arg("codes_a"), py::arg("codes_b"));
}
