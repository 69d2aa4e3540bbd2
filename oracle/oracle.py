"""ctypes front-end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs
import this module.  It wraps:

* ``liboracle.so`` -- the plain-C restatement (tq_oracle.c) of the reference's
  encode-and-scan path (include/turboquant/space_turbo_quant.h:339-615);
* ``_ref/libtqref.so`` and ``_ref/_turboquant*.so`` -- the reference library
  itself, compiled here from its own sources by ``make ref``.  They are
  optional: where they are absent the restatement is the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_sz = C.c_size_t


def _f32(a):
    return a.ctypes.data_as(_fp)


def _u8(a):
    return a.ctypes.data_as(_u8p)


def build_oracle() -> str:
    """Compile liboracle.so in place if it is missing; return its path."""
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return path


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(build_oracle())
        L.tqo_create.restype = C.c_void_p
        L.tqo_create.argtypes = [_sz, C.c_int, C.c_uint64, C.c_uint64]
        L.tqo_destroy.argtypes = [C.c_void_p]
        L.tqo_space_padded_dim.restype = _sz
        L.tqo_space_padded_dim.argtypes = [C.c_void_p]
        L.tqo_space_code_size.restype = _sz
        L.tqo_space_code_size.argtypes = [C.c_void_p]
        L.tqo_space_scale.restype = C.c_float
        L.tqo_space_scale.argtypes = [C.c_void_p]
        for nm in ("centroids", "boundaries", "rot_signs", "qjl_signs"):
            f = getattr(L, "tqo_space_" + nm)
            f.restype = _fp
            f.argtypes = [C.c_void_p]
        L.tqo_sq_reduce.restype = C.c_float
        L.tqo_sq_reduce.argtypes = [_fp, _sz]
        L.tqo_lloyd_max.argtypes = [C.c_int, _fp, _fp]
        L.tqo_signs.argtypes = [_sz, C.c_uint64, _fp]
        L.tqo_encode_batch.argtypes = [C.c_void_p, _fp, _sz, _u8p, C.c_int]
        L.tqo_prepare_query.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp]
        L.tqo_distance_1_to_n.argtypes = [C.c_void_p, _fp, _u8p, _sz, _fp, C.c_int]
        L.tqo_distance_m_to_n.argtypes = [C.c_void_p, _fp, _sz, _u8p, _sz, _fp, C.c_int]
        L.tqo_distance_m_to_n_symmetric.argtypes = [C.c_void_p, _u8p, _sz, _u8p, _sz, _fp,
                                                    C.c_int]
        L.tqo_distance_f64.restype = C.c_double
        L.tqo_distance_f64.argtypes = [C.c_void_p, _fp, _u8p]
        L.tqo_distance_symmetric_f64.restype = C.c_double
        L.tqo_distance_symmetric_f64.argtypes = [C.c_void_p, _u8p, _u8p]
        L.tqo_rotated_coords_batch.argtypes = [C.c_void_p, _fp, _sz, _fp, C.c_int]
        L.tqo_distance_m_to_n_symmetric_qjl.argtypes = [C.c_void_p, _u8p, _sz, _u8p, _sz, _fp,
                                                        C.c_int, C.c_int]
        L.tqo_prepare_symmetric.argtypes = [C.c_void_p, _u8p, _fp, _fp, _fp]
        L.tqo_distance_1_to_n_symmetric_full.argtypes = [C.c_void_p, _fp, _fp, _fp, _u8p, _sz,
                                                         _fp, C.c_int]
        L.tqo_distance_symmetric_qjl_f64.restype = C.c_double
        L.tqo_distance_symmetric_qjl_f64.argtypes = [C.c_void_p, _u8p, _u8p, C.c_int]
        _LIB = L
    return _LIB


def _threads(n):
    return n if n and n > 0 else (os.cpu_count() or 1)


class OracleSpace:
    """The restatement, shaped like the reference's TurboQuantSpace."""

    def __init__(self, dim, bits_per_coord=4, rot_seed=42, qjl_seed=137, num_threads=0):
        self._L = lib()
        self._h = self._L.tqo_create(dim, bits_per_coord, rot_seed, qjl_seed)
        if not self._h:
            raise ValueError("invalid space parameters")
        self.dim_ = int(dim)
        self.bits = int(bits_per_coord)
        self.D = int(self._L.tqo_space_padded_dim(self._h))
        self.cs = int(self._L.tqo_space_code_size(self._h))
        self.threads = _threads(num_threads)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.tqo_destroy(h)
            self._h = None

    # geometry / tables
    def dim(self):
        return self.dim_

    def padded_dim(self):
        return self.D

    def code_size_bytes(self):
        return self.cs

    def scale(self):
        return float(self._L.tqo_space_scale(self._h))

    def tables(self):
        L = 1 << (self.bits - 1)
        c = np.ctypeslib.as_array(self._L.tqo_space_centroids(self._h), (L,)).copy()
        b = np.ctypeslib.as_array(self._L.tqo_space_boundaries(self._h), (max(L - 1, 1),))[:L - 1].copy()
        rs = np.ctypeslib.as_array(self._L.tqo_space_rot_signs(self._h), (self.D,)).copy()
        qs = np.ctypeslib.as_array(self._L.tqo_space_qjl_signs(self._h), (self.D,)).copy()
        return c, b, rs, qs

    # path
    def encode_batch(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        n = X.shape[0]
        out = np.empty((n, self.cs), dtype=np.uint8)
        self._L.tqo_encode_batch(self._h, _f32(X), n, _u8(out), self.threads)
        return out

    def prepare_query(self, q):
        q = np.ascontiguousarray(q, dtype=np.float32)
        q_rot = np.empty(self.D, np.float32)
        s_q = np.empty(self.D, np.float32)
        norms = np.empty(2, np.float32)
        self._L.tqo_prepare_query(self._h, _f32(q), _f32(q_rot), _f32(s_q), _f32(norms))
        return q_rot, s_q, norms

    def distance_1_to_n(self, q, codes):
        q = np.ascontiguousarray(q, dtype=np.float32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        n = codes.size // self.cs
        out = np.empty(n, np.float32)
        self._L.tqo_distance_1_to_n(self._h, _f32(q), _u8(codes), n, _f32(out), self.threads)
        return out

    def distance_m_to_n(self, Q, codes):
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        m, n = Q.shape[0], codes.size // self.cs
        out = np.empty((m, n), np.float32)
        self._L.tqo_distance_m_to_n(self._h, _f32(Q), m, _u8(codes), n, _f32(out), self.threads)
        return out

    def distance_m_to_n_symmetric(self, A, B):
        A = np.ascontiguousarray(A, dtype=np.uint8)
        B = np.ascontiguousarray(B, dtype=np.uint8)
        m, n = A.size // self.cs, B.size // self.cs
        out = np.empty((m, n), np.float32)
        self._L.tqo_distance_m_to_n_symmetric(self._h, _u8(A), m, _u8(B), n, _f32(out),
                                              self.threads)
        return out

    def distance_f64(self, q, code):
        q = np.ascontiguousarray(q, dtype=np.float32)
        code = np.ascontiguousarray(code, dtype=np.uint8)
        return float(self._L.tqo_distance_f64(self._h, _f32(q), _u8(code)))

    def distance_symmetric_f64(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.uint8)
        b = np.ascontiguousarray(b, dtype=np.uint8)
        return float(self._L.tqo_distance_symmetric_f64(self._h, _u8(a), _u8(b)))


    # rotatedCoordsBatch and the QJL-corrected symmetric distances
    SYM_VARIANTS = {"light": 0, "full": 1, "full_prepared": 2}

    def rotated_coords_batch(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty((X.shape[0], self.D), np.float32)
        self._L.tqo_rotated_coords_batch(self._h, _f32(X), X.shape[0], _f32(out), self.threads)
        return out

    def distance_m_to_n_symmetric_qjl(self, A, B, variant):
        A = np.ascontiguousarray(A, dtype=np.uint8)
        B = np.ascontiguousarray(B, dtype=np.uint8)
        m, n = A.size // self.cs, B.size // self.cs
        out = np.empty((m, n), np.float32)
        self._L.tqo_distance_m_to_n_symmetric_qjl(self._h, _u8(A), m, _u8(B), n, _f32(out),
                                                  self.SYM_VARIANTS[variant], self.threads)
        return out

    def prepare_symmetric_query(self, code):
        code = np.ascontiguousarray(code, dtype=np.uint8)
        recon = np.empty(self.D, np.float32)
        sign = np.empty(self.D, np.float32)
        sc = np.empty(5, np.float32)
        self._L.tqo_prepare_symmetric(self._h, _u8(code), _f32(recon), _f32(sign), _f32(sc))
        return recon, sign, sc

    def distance_1_to_n_symmetric_full(self, prepared, codes):
        recon, sign, sc = (np.ascontiguousarray(a, dtype=np.float32) for a in prepared)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        n = codes.size // self.cs
        out = np.empty(n, np.float32)
        self._L.tqo_distance_1_to_n_symmetric_full(self._h, _f32(recon), _f32(sign), _f32(sc),
                                                   _u8(codes), n, _f32(out), self.threads)
        return out

    def distance_symmetric_qjl_f64(self, a, b, variant):
        a = np.ascontiguousarray(a, dtype=np.uint8)
        b = np.ascontiguousarray(b, dtype=np.uint8)
        return float(self._L.tqo_distance_symmetric_qjl_f64(self._h, _u8(a), _u8(b),
                                                            self.SYM_VARIANTS[variant]))


def sq_reduce(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    return float(lib().tqo_sq_reduce(_f32(x), x.size))


# --------------------------------------------------------------------------
# The reference itself, compiled from its sources (optional).
# --------------------------------------------------------------------------
_REFLIB = None


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libtqref.so"))


def ref_lib():
    global _REFLIB
    if _REFLIB is None:
        L = C.CDLL(os.path.join(REF_DIR, "libtqref.so"))
        L.tqr_create.restype = C.c_void_p
        L.tqr_create.argtypes = [_sz, C.c_int, C.c_uint64, C.c_uint64, C.c_int]
        L.tqr_destroy.argtypes = [C.c_void_p]
        L.tqr_code_size.restype = _sz
        L.tqr_code_size.argtypes = [C.c_void_p]
        L.tqr_padded_dim.restype = _sz
        L.tqr_padded_dim.argtypes = [C.c_void_p]
        L.tqr_scale.restype = C.c_float
        L.tqr_scale.argtypes = [C.c_void_p]
        L.tqr_tables.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp]
        L.tqr_encode_batch.argtypes = [C.c_void_p, _fp, _sz, _u8p]
        L.tqr_prepare_query.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp]
        L.tqr_distance_1_to_n.argtypes = [C.c_void_p, _fp, _u8p, _sz, _fp]
        L.tqr_distance_m_to_n.argtypes = [C.c_void_p, _fp, _sz, _u8p, _sz, _fp]
        L.tqr_distance_m_to_n_symmetric.argtypes = [C.c_void_p, _u8p, _sz, _u8p, _sz, _fp]
        _REFLIB = L
    return _REFLIB


class RefSpace:
    """The reference's TurboQuantSpace through the C shim (oracle/ref_shim.cpp)."""

    def __init__(self, dim, bits_per_coord=4, rot_seed=42, qjl_seed=137, num_threads=0):
        self._L = ref_lib()
        self._h = self._L.tqr_create(dim, bits_per_coord, rot_seed, qjl_seed, num_threads)
        self.dim_ = int(dim)
        self.bits = int(bits_per_coord)
        self.D = int(self._L.tqr_padded_dim(self._h))
        self.cs = int(self._L.tqr_code_size(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.tqr_destroy(h)
            self._h = None

    def scale(self):
        return float(self._L.tqr_scale(self._h))

    def tables(self):
        L = 1 << (self.bits - 1)
        c = np.empty(L, np.float32)
        b = np.empty(max(L - 1, 1), np.float32)
        rs = np.empty(self.D, np.float32)
        qs = np.empty(self.D, np.float32)
        self._L.tqr_tables(self._h, _f32(c), _f32(b), _f32(rs), _f32(qs))
        return c, b[:L - 1], rs, qs

    def encode_batch(self, X):
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty((X.shape[0], self.cs), np.uint8)
        self._L.tqr_encode_batch(self._h, _f32(X), X.shape[0], _u8(out))
        return out

    def prepare_query(self, q):
        q = np.ascontiguousarray(q, dtype=np.float32)
        q_rot = np.empty(self.D, np.float32)
        s_q = np.empty(self.D, np.float32)
        norms = np.empty(2, np.float32)
        self._L.tqr_prepare_query(self._h, _f32(q), _f32(q_rot), _f32(s_q), _f32(norms))
        return q_rot, s_q, norms

    def distance_1_to_n(self, q, codes):
        q = np.ascontiguousarray(q, dtype=np.float32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        n = codes.size // self.cs
        out = np.empty(n, np.float32)
        self._L.tqr_distance_1_to_n(self._h, _f32(q), _u8(codes), n, _f32(out))
        return out

    def distance_m_to_n(self, Q, codes):
        Q = np.ascontiguousarray(Q, dtype=np.float32)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        m, n = Q.shape[0], codes.size // self.cs
        out = np.empty((m, n), np.float32)
        self._L.tqr_distance_m_to_n(self._h, _f32(Q), m, _u8(codes), n, _f32(out))
        return out

    def distance_m_to_n_symmetric(self, A, B):
        A = np.ascontiguousarray(A, dtype=np.uint8)
        B = np.ascontiguousarray(B, dtype=np.uint8)
        m, n = A.size // self.cs, B.size // self.cs
        out = np.empty((m, n), np.float32)
        self._L.tqr_distance_m_to_n_symmetric(self._h, _u8(A), m, _u8(B), n, _f32(out))
        return out


def import_ref_module():
    """The reference's own pybind11 module (_turboquant), built by ``make ref``."""
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import _turboquant  # noqa: E402
    return _turboquant
