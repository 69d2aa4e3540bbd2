"""turboquant -- TurboQuant encode-and-scan on B200 (sm_100a).

A drop-in for the reference package's ``TurboQuantSpace``
(python/turboquant/__init__.py, bindings.cpp:53-218 of ilyajob05/turboquant-space):
the same constructor, method names, keyword names, defaults, output shapes and
``ValueError`` texts, with the work done by libtqb200.so's CUDA kernels.

Inputs may be any buffer-protocol object (as with the reference's
``py::buffer``) -- those run through the synchronous host-pointer entry points
-- or CUDA arrays exposing ``__cuda_array_interface__`` or ``__dlpack__``
(torch, CuPy, JAX, ...), which run stream-ordered on torch's current stream and
return torch CUDA tensors.  ``load_codes`` streams a code file (.npy or raw)
into HBM.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import TQError, check, lib

__all__ = ["TurboQuantSpace", "PreparedQuery", "PreparedSymCode", "TQError", "Index", "Server",
           "BusyError", "load_codes"]
__version__ = "0.1.0"


# ---------------------------------------------------------------------------
# argument validation, mirroring bindings.cpp:14-49
# ---------------------------------------------------------------------------
def _dlpack_cuda(obj) -> bool:
    """A DLPack producer (``__dlpack__``) whose memory is on a CUDA device."""
    if hasattr(obj, "__cuda_array_interface__") or not hasattr(obj, "__dlpack_device__"):
        return False
    try:
        return int(obj.__dlpack_device__()[0]) in (2, 13)  # kDLCUDA, kDLCUDAManaged
    except Exception:  # a producer that cannot answer is not a device array
        return False


def _is_device(obj) -> bool:
    return hasattr(obj, "__cuda_array_interface__") or _dlpack_cuda(obj)


def _as_cai(obj):
    """The object itself if it exposes ``__cuda_array_interface__``, else a
    zero-copy torch view of a CUDA DLPack producer (torch.from_dlpack passes
    torch's current stream, so the producer's pending work is ordered first)."""
    if hasattr(obj, "__cuda_array_interface__"):
        return obj
    return _torch().utils.dlpack.from_dlpack(obj)


def _float_host(buf, expected_last, name, expected_ndim):
    """as_float_ptr (bindings.cpp:14-36). Returns a C-contiguous float32 ndarray.

    The reference checks only the innermost stride; rows that are not packed
    would be read as if they were.  Here such rows are gathered into a packed
    copy, so the result is the one the caller meant."""
    mv = memoryview(buf)
    if mv.format not in ("f", "<f", "=f"):
        raise ValueError(f"{name}: expected float32")
    if mv.ndim != expected_ndim:
        raise ValueError(f"{name}: wrong ndim")
    if expected_ndim == 1:
        if mv.shape[0] != expected_last:
            raise ValueError(f"{name}: wrong length")
    else:
        if mv.shape[1] != expected_last:
            raise ValueError(f"{name}: wrong dim")
    if mv.strides[mv.ndim - 1] != 4:
        raise ValueError(f"{name}: must be C-contiguous float32")
    return np.ascontiguousarray(np.asarray(mv).view(np.float32))


def _bytes_host(buf, name, writable):
    mv = memoryview(buf)
    if writable and mv.readonly:
        raise BufferError("Writable buffer requested for readonly storage")
    if mv.itemsize != 1:
        raise ValueError(f"{name}: must be uint8")
    return mv


def _codes_host(buf, cs, bad_type_msg="codes must be uint8"):
    """codes argument of the batch distances (bindings.cpp:159-167)."""
    mv = memoryview(buf)
    if mv.itemsize != 1:
        raise ValueError(bad_type_msg)
    total = mv.nbytes
    if total % cs != 0:
        raise ValueError("codes size not a multiple of code_size_bytes")
    arr = np.ascontiguousarray(np.asarray(mv).view(np.uint8)).reshape(-1)
    return arr, total // cs


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _out_host(out, shape):
    """Optional caller-provided result buffer (an extension of the reference
    API): a writable C-contiguous float32 array of exactly ``shape``."""
    if out is None:
        return np.empty(shape, np.float32)
    arr = np.asarray(out)
    if arr.dtype != np.float32 or arr.shape != tuple(shape) or not arr.flags.c_contiguous \
            or not arr.flags.writeable:
        raise ValueError(f"out: expected a writable C-contiguous float32 array of shape {shape}")
    return arr


# ---------------------------------------------------------------------------
# CUDA array helpers (torch is the plumbing for device memory and streams)
# ---------------------------------------------------------------------------
def _torch():
    import torch  # noqa: WPS433 - imported lazily: only device inputs need it
    return torch


def _cai(obj):
    cai = _as_cai(obj).__cuda_array_interface__
    shape = tuple(cai["shape"])
    typestr = cai["typestr"]
    strides = cai.get("strides")
    ptr = cai["data"][0]
    return ptr, shape, typestr, strides


def _contig(shape, strides, itemsize):
    if strides is None:
        return True
    expect = itemsize
    for dim, st in zip(reversed(shape), reversed(strides)):
        if dim != 1 and st != expect:
            return False
        expect *= dim
    return True


def _float_dev(obj, expected_last, name, expected_ndim):
    ptr, shape, typestr, strides = _cai(obj)
    if typestr not in ("<f4", "=f4", "f4"):
        raise ValueError(f"{name}: expected float32")
    if len(shape) != expected_ndim:
        raise ValueError(f"{name}: wrong ndim")
    if expected_ndim == 1 and shape[0] != expected_last:
        raise ValueError(f"{name}: wrong length")
    if expected_ndim == 2 and shape[1] != expected_last:
        raise ValueError(f"{name}: wrong dim")
    if not _contig(shape, strides, 4):
        raise ValueError(f"{name}: must be C-contiguous float32")
    return ptr, shape


def _codes_dev(obj, cs, bad_type_msg="codes must be uint8"):
    ptr, shape, typestr, strides = _cai(obj)
    if typestr[-1] != "1":
        raise ValueError(bad_type_msg)
    total = int(np.prod(shape)) if shape else 1
    if total % cs != 0:
        raise ValueError("codes size not a multiple of code_size_bytes")
    if not _contig(shape, strides, 1):
        raise ValueError("codes must be contiguous")
    return ptr, total // cs


def _stream_and_device(obj):
    torch = _torch()
    obj = _as_cai(obj)
    dev = obj.device if isinstance(getattr(obj, "device", None), torch.device) \
        else torch.device("cuda", torch.cuda.current_device())
    return torch.cuda.current_stream(dev).cuda_stream, dev


class PreparedQuery:
    """TurboQuantPreparedQuery (space_turbo_quant.h:138-144): a query rotated
    once (q_rot = RHT_rot(q / |q|)), its QJL image (s_q = RHT_qjl(q_rot)) and
    its norms, held on the host as float32.  The reference binds it as an
    opaque object (bindings.cpp:56); its fields are exposed here."""

    __slots__ = ("q_rot", "s_q", "q_norm_sq", "q_norm")

    def __init__(self, q_rot, s_q, q_norm_sq, q_norm):
        self.q_rot = np.ascontiguousarray(q_rot, dtype=np.float32)
        self.s_q = np.ascontiguousarray(s_q, dtype=np.float32)
        self.q_norm_sq = float(q_norm_sq)
        self.q_norm = float(q_norm)


class PreparedSymCode:
    """TurboQuantPreparedSymCode (space_turbo_quant.h:158-166): one code
    reconstructed and passed through the QJL Hadamard (recon_q), its +-1 QJL
    signs (sign_q) and the scalars [norm, gamma, sigma, scale * gamma,
    (pi / 2D) * gamma], held on the host as float32 arrays."""

    __slots__ = ("recon_q", "sign_q", "scalars")

    def __init__(self, recon_q, sign_q, scalars):
        self.recon_q = np.ascontiguousarray(recon_q, dtype=np.float32)
        self.sign_q = np.ascontiguousarray(sign_q, dtype=np.float32)
        self.scalars = np.ascontiguousarray(scalars, dtype=np.float32)

    @property
    def norm_q(self):
        return float(self.scalars[0])

    @property
    def gamma_q(self):
        return float(self.scalars[1])

    @property
    def sigma_q(self):
        return float(self.scalars[2])


class TurboQuantSpace:
    """TurboQuant space (space_turbo_quant.h:207-648) on one GPU.

    ``TurboQuantSpace(dim, bits_per_coord=4, rot_seed=42, qjl_seed=137,
    num_threads=0)`` as in bindings.cpp:60-65; ``device`` (keyword only)
    selects the CUDA device (default: the current one)."""

    def __init__(self, dim, bits_per_coord=4, rot_seed=42, qjl_seed=137, num_threads=0, *,
                 device=-1):
        dim = int(dim)
        if dim < 0:
            raise TypeError("dim must be a non-negative integer")
        if num_threads is None or int(num_threads) <= 0:
            env = os.environ.get("OMP_NUM_THREADS", "")
            num_threads = int(env) if env.isdigit() and int(env) > 0 else (os.cpu_count() or 1)
        h = C.c_void_p()
        check(lib().tq_space_create(dim, int(bits_per_coord), int(rot_seed) & (2**64 - 1),
                                    int(qjl_seed) & (2**64 - 1), int(num_threads), int(device),
                                    C.byref(h)))
        self._h = h
        info = _capi.SpaceInfo()
        check(lib().tq_space_get_info(self._h, C.byref(info)))
        self._info = info

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().tq_space_destroy(h)
            except Exception:  # interpreter teardown
                pass
            self._h = None

    # -- accessors (bindings.cpp:67-72) ------------------------------------
    def dim(self):
        return int(self._info.dim)

    def padded_dim(self):
        return int(self._info.padded_dim)

    def padded(self):
        return bool(self._info.padded)

    def num_threads(self):
        return int(self._info.num_threads)

    def code_size_bytes(self):
        return int(self._info.code_size)

    def bits_per_coord(self):
        return int(self._info.bits_per_coord)

    # extras (TurboQuantSpace accessors the binding does not expose)
    def packed_bytes(self):
        return int(self._info.packed_bytes)

    def scale(self):
        return float(self._info.scale)

    def device(self):
        return int(self._info.device)

    def tables(self):
        """(centroids, boundaries, rot_signs, qjl_signs) as float32 arrays."""
        L = int(self._info.num_levels)
        D = self.padded_dim()
        c = np.empty(L, np.float32)
        b = np.empty(max(L - 1, 1), np.float32)
        r = np.empty(D, np.float32)
        q = np.empty(D, np.float32)
        check(lib().tq_space_tables(self._h, _ptr(c), _ptr(b), _ptr(r), _ptr(q)))
        return c, b[:L - 1], r, q

    def quantize(self, z):
        """Host-side quantize of normalised values through the encode kernel's
        bucket table (a diagnostic; space_turbo_quant.h:332-337)."""
        z = np.ascontiguousarray(z, dtype=np.float32).reshape(-1)
        idx = np.empty(z.size, np.uint8)
        check(lib().tq_space_quantize(self._h, _ptr(z), z.size, _ptr(idx)))
        return idx

    # -- encode (bindings.cpp:75-116) ----------------------------------------
    def encode(self, x):
        data = _float_host(x, self.dim(), "input", 1)
        code = np.empty(self.code_size_bytes(), np.uint8)
        check(lib().tq_encode_batch(self._h, _ptr(data), 1, _ptr(code)))
        return code

    def encode_into(self, x, out):
        data = _float_host(x, self.dim(), "input", 1)
        mv = _bytes_host(out, "code", True)
        if mv.nbytes != self.code_size_bytes():
            raise ValueError("code: wrong byte size")
        tmp = np.empty(self.code_size_bytes(), np.uint8)
        check(lib().tq_encode_batch(self._h, _ptr(data), 1, _ptr(tmp)))
        np.asarray(mv).reshape(-1).view(np.uint8)[:] = tmp

    def encode_batch(self, X):
        if _is_device(X):
            ptr, shape = _float_dev(X, self.dim(), "input", 2)
            torch = _torch()
            stream, dev = _stream_and_device(X)
            out = torch.empty((shape[0], self.code_size_bytes()), dtype=torch.uint8, device=dev)
            check(lib().tq_encode_batch_device(self._h, C.c_void_p(ptr), shape[0],
                                               C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
            return out
        data = _float_host(X, self.dim(), "input", 2)
        n = data.shape[0]
        codes = np.empty((n, self.code_size_bytes()), np.uint8)
        check(lib().tq_encode_batch(self._h, _ptr(data), n, _ptr(codes)))
        return codes

    def encode_batch_into(self, X, out):
        if _is_device(X):
            ptr, shape = _float_dev(X, self.dim(), "input", 2)
            optr, nbytes = _codes_dev(out, 1)
            if nbytes != shape[0] * self.code_size_bytes():
                raise ValueError("codes: wrong byte size")
            stream, _ = _stream_and_device(X)
            check(lib().tq_encode_batch_device(self._h, C.c_void_p(ptr), shape[0],
                                               C.c_void_p(optr), C.c_void_p(stream)))
            return None
        data = _float_host(X, self.dim(), "input", 2)
        n = data.shape[0]
        mv = _bytes_host(out, "codes", True)
        if mv.nbytes != n * self.code_size_bytes():
            raise ValueError("codes: wrong byte size")
        target = np.asarray(mv).reshape(-1).view(np.uint8)
        if target.flags.c_contiguous:
            check(lib().tq_encode_batch(self._h, _ptr(data), n, _ptr(target)))
        else:
            tmp = np.empty(n * self.code_size_bytes(), np.uint8)
            check(lib().tq_encode_batch(self._h, _ptr(data), n, _ptr(tmp)))
            target[:] = tmp
        return None

    # -- single distances (bindings.cpp:135-153) ----------------------------
    def distance(self, query, code):
        q = _float_host(query, self.dim(), "query", 1)
        mv = _bytes_host(code, "code", False)
        if mv.nbytes != self.code_size_bytes():
            raise ValueError("code: wrong byte size")
        c = np.ascontiguousarray(np.asarray(mv).reshape(-1).view(np.uint8))
        out = np.empty(1, np.float32)
        check(lib().tq_distance_1_to_n(self._h, _ptr(q), _ptr(c), 1, _ptr(out)))
        return float(out[0])

    def distance_symmetric(self, code_a, code_b):
        cs = self.code_size_bytes()
        mva = _bytes_host(code_a, "code_a", False)
        if mva.nbytes != cs:
            raise ValueError("code_a: wrong byte size")
        mvb = _bytes_host(code_b, "code_b", False)
        if mvb.nbytes != cs:
            raise ValueError("code_b: wrong byte size")
        a = np.ascontiguousarray(np.asarray(mva).reshape(-1).view(np.uint8))
        b = np.ascontiguousarray(np.asarray(mvb).reshape(-1).view(np.uint8))
        out = np.empty(1, np.float32)
        check(lib().tq_distance_m_to_n_symmetric(self._h, _ptr(a), 1, _ptr(b), 1, _ptr(out), 0))
        return float(out[0])

    # -- batch distances (bindings.cpp:156-218) ------------------------------
    def distance_1_to_n(self, query, codes, out=None):
        cs = self.code_size_bytes()
        if _is_device(query) or _is_device(codes):
            qptr, _ = _float_dev(query, self.dim(), "query", 1)
            cptr, n = _codes_dev(codes, cs)
            torch = _torch()
            stream, dev = _stream_and_device(codes)
            out = torch.empty(n, dtype=torch.float32, device=dev)
            check(lib().tq_distance_1_to_n_device(self._h, C.c_void_p(qptr), C.c_void_p(cptr), n,
                                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
            return out
        q = _float_host(query, self.dim(), "query", 1)
        c, n = _codes_host(codes, cs)
        out = _out_host(out, (n,))
        check(lib().tq_distance_1_to_n(self._h, _ptr(q), _ptr(c), n, _ptr(out)))
        return out

    def distance_m_to_n(self, queries, codes, precision="fp32", out=None):
        """distanceBatchMToN: queries [m, dim] float32 x codes [n, cs] -> [m, n].

        precision: "fp32" (CUDA cores, the drop-in), "split_bf16" (tcgen05
        tensor cores on hi+lo BF16 operand planes), "split_bf16_decoded" (the
        same arithmetic, column tiles decoded from the codes in shared memory:
        less device memory, somewhat slower) or "reference" (the reference
        build's own summation order, bit-identical distances)."""
        cs = self.code_size_bytes()
        prec = _capi.PRECISION[precision]
        if _is_device(queries) or _is_device(codes):
            qptr, shape = _float_dev(queries, self.dim(), "queries", 2)
            cptr, n = _codes_dev(codes, cs)
            torch = _torch()
            stream, dev = _stream_and_device(codes)
            out = torch.empty((shape[0], n), dtype=torch.float32, device=dev)
            check(lib().tq_distance_m_to_n_device(self._h, C.c_void_p(qptr), shape[0],
                                                  C.c_void_p(cptr), n, C.c_void_p(out.data_ptr()),
                                                  prec, C.c_void_p(stream)))
            return out
        q = _float_host(queries, self.dim(), "queries", 2)
        c, n = _codes_host(codes, cs)
        m = q.shape[0]
        out = _out_host(out, (m, n))
        check(lib().tq_distance_m_to_n(self._h, _ptr(q), m, _ptr(c), n, _ptr(out), prec))
        return out

    def distance_m_to_n_symmetric(self, codes_a, codes_b, precision="fp32", out=None):
        """distanceBatchMToNSymmetric: codes_a [m, cs] x codes_b [n, cs] -> [m, n].

        precision: "fp32", "split_bf16", "split_bf16_decoded" or "reference",
        as for distance_m_to_n."""
        cs = self.code_size_bytes()
        prec = _capi.PRECISION[precision]
        if _is_device(codes_a) or _is_device(codes_b):
            aptr, m = _codes_dev(codes_a, cs)
            bptr, n = _codes_dev(codes_b, cs)
            torch = _torch()
            stream, dev = _stream_and_device(codes_b)
            out = torch.empty((m, n), dtype=torch.float32, device=dev)
            check(lib().tq_distance_m_to_n_symmetric_device(
                self._h, C.c_void_p(aptr), m, C.c_void_p(bptr), n, C.c_void_p(out.data_ptr()),
                prec, C.c_void_p(stream)))
            return out
        mva, mvb = memoryview(codes_a), memoryview(codes_b)
        if mva.itemsize != 1 or mvb.itemsize != 1:
            raise ValueError("codes must be uint8")
        if mva.nbytes % cs != 0 or mvb.nbytes % cs != 0:
            raise ValueError("codes size not a multiple of code_size_bytes")
        a, m = _codes_host(codes_a, cs)
        b, n = _codes_host(codes_b, cs)
        out = _out_host(out, (m, n))
        check(lib().tq_distance_m_to_n_symmetric(self._h, _ptr(a), m, _ptr(b), n, _ptr(out), prec))
        return out

    # -- rotated coordinates (bindings.cpp:119-132) ---------------------------
    def rotated_coords_batch(self, X):
        """(n, padded_dim) sigma-normalised post-rotation coordinates
        (rotatedCoordsBatch, space_turbo_quant.h:411-435), bit-identical."""
        D = self.padded_dim()
        if _is_device(X):
            ptr, shape = _float_dev(X, self.dim(), "input", 2)
            torch = _torch()
            stream, dev = _stream_and_device(X)
            out = torch.empty((shape[0], D), dtype=torch.float32, device=dev)
            check(lib().tq_rotated_coords_batch_device(self._h, C.c_void_p(ptr), shape[0],
                                                       C.c_void_p(out.data_ptr()),
                                                       C.c_void_p(stream)))
            return out
        data = _float_host(X, self.dim(), "input", 2)
        out = np.empty((data.shape[0], D), np.float32)
        check(lib().tq_rotated_coords_batch(self._h, _ptr(data), data.shape[0], _ptr(out)))
        return out

    # -- QJL-corrected symmetric distances (bindings.cpp:221-334) --------------
    def _symmetric_qjl(self, codes_a, codes_b, variant, precision):
        cs = self.code_size_bytes()
        v = _capi.SYM_VARIANT[variant]
        prec = _capi.PRECISION[precision]
        if _is_device(codes_a) or _is_device(codes_b):
            aptr, m = _codes_dev(codes_a, cs)
            bptr, n = _codes_dev(codes_b, cs)
            torch = _torch()
            stream, dev = _stream_and_device(codes_b)
            out = torch.empty((m, n), dtype=torch.float32, device=dev)
            check(lib().tq_distance_m_to_n_symmetric_qjl_device(
                self._h, C.c_void_p(aptr), m, C.c_void_p(bptr), n, C.c_void_p(out.data_ptr()), v,
                prec, C.c_void_p(stream)))
            return out
        mva, mvb = memoryview(codes_a), memoryview(codes_b)
        if mva.itemsize != 1 or mvb.itemsize != 1:
            raise ValueError("codes must be uint8")
        if mva.nbytes % cs != 0 or mvb.nbytes % cs != 0:
            raise ValueError("codes size not a multiple of code_size_bytes")
        a, m = _codes_host(codes_a, cs)
        b, n = _codes_host(codes_b, cs)
        out = np.empty((m, n), np.float32)
        check(lib().tq_distance_m_to_n_symmetric_qjl(self._h, _ptr(a), m, _ptr(b), n, _ptr(out), v,
                                                     prec))
        return out

    # precision="fp32" is the drop-in (CUDA cores); "split_tf32" runs the two
    # contractions on tcgen05 tensor cores (hi/lo TF32 operands, FP32 sums).
    def distance_m_to_n_symmetric_full(self, codes_a, codes_b, precision="fp32"):
        """distanceBatchMToNSymmetricFull: MSE + all four QJL terms (:618-631, 731-800)."""
        return self._symmetric_qjl(codes_a, codes_b, "full", precision)

    def distance_m_to_n_symmetric_light(self, codes_a, codes_b, precision="fp32"):
        """distanceBatchMToNSymmetricLight: MSE + the sign-agreement term (:634-647, 902-945)."""
        return self._symmetric_qjl(codes_a, codes_b, "light", precision)

    def distance_m_to_n_symmetric_full_prepared(self, codes_a, codes_b, precision="fp32"):
        """distanceBatchMToNSymmetricFullPrepared: row codes prepared once (:557-572, 808-878)."""
        return self._symmetric_qjl(codes_a, codes_b, "full_prepared", precision)

    def prepare_query(self, query):
        """prepareQuery (:439-460; bindings.cpp:268-273) of one query: a PreparedQuery."""
        q = _float_host(query, self.dim(), "query", 1)
        D = self.padded_dim()
        q_rot = np.empty(D, np.float32)
        s_q = np.empty(D, np.float32)
        norms = np.empty(2, np.float32)
        check(lib().tq_prepare_query(self._h, _ptr(q), _ptr(q_rot), _ptr(s_q), _ptr(norms)))
        return PreparedQuery(q_rot, s_q, norms[0], norms[1])

    def prepare_symmetric_query(self, code):
        """prepareSymmetricQuery (:499-535) of one code: a PreparedSymCode."""
        mv = _bytes_host(code, "code", False)
        if mv.nbytes != self.code_size_bytes():
            raise ValueError("code: wrong byte size")
        c = np.ascontiguousarray(np.asarray(mv).reshape(-1).view(np.uint8))
        D = self.padded_dim()
        recon = np.empty(D, np.float32)
        sign = np.empty(D, np.float32)
        sc = np.empty(5, np.float32)
        check(lib().tq_prepare_symmetric_query(self._h, _ptr(c), _ptr(recon), _ptr(sign), _ptr(sc)))
        return PreparedSymCode(recon, sign, sc)

    def distance_symmetric_full_prepared(self, pq, code_b):
        """distanceSymmetricFullPrepared (:538-541): one prepared code x one code."""
        mv = _bytes_host(code_b, "code_b", False)
        if mv.nbytes != self.code_size_bytes():
            raise ValueError("code_b: wrong byte size")
        b = np.ascontiguousarray(np.asarray(mv).reshape(-1).view(np.uint8))
        return float(self.distance_1_to_n_symmetric_full(pq, b)[0])

    def distance_1_to_n_symmetric_full(self, pq, codes):
        """distanceBatch1ToNSymmetricFull (:544-553): a prepared code x n codes."""
        if not isinstance(pq, PreparedSymCode):
            raise TypeError("pq: expected a PreparedSymCode")
        cs = self.code_size_bytes()
        if _is_device(codes):
            cptr, n = _codes_dev(codes, cs)
            torch = _torch()
            stream, dev = _stream_and_device(codes)
            r = torch.from_numpy(pq.recon_q).to(dev)
            sg = torch.from_numpy(pq.sign_q).to(dev)
            sc = torch.from_numpy(pq.scalars).to(dev)
            out = torch.empty(n, dtype=torch.float32, device=dev)
            check(lib().tq_distance_1_to_n_symmetric_full_device(
                self._h, C.c_void_p(r.data_ptr()), C.c_void_p(sg.data_ptr()),
                C.c_void_p(sc.data_ptr()), C.c_void_p(cptr), n, C.c_void_p(out.data_ptr()),
                C.c_void_p(stream)))
            return out
        c, n = _codes_host(codes, cs)
        out = np.empty(n, np.float32)
        check(lib().tq_distance_1_to_n_symmetric_full(self._h, _ptr(pq.recon_q), _ptr(pq.sign_q),
                                                      _ptr(pq.scalars), _ptr(c), n, _ptr(out)))
        return out

    def index(self, codes, layout="planes"):
        """A device-resident search index over `codes` (see turboquant.serving)."""
        return Index(self, codes, layout)

    def __repr__(self):
        return (f"TurboQuantSpace(dim={self.dim()}, bits_per_coord={self.bits_per_coord()}, "
                f"padded_dim={self.padded_dim()}, code_size_bytes={self.code_size_bytes()}, "
                f"device={self.device()})")


from .serving import BusyError, Index, Server, variant_shapes  # noqa: E402
from .io import load_codes  # noqa: E402
