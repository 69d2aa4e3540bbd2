"""Device-resident index and continuous-batching top-k server (libtqb200).

The reference has no index or serving loop (its README.md:81-83); this wraps
the C ABI's tq_index_* / tq_server_* entry points:

    index = Index(space, codes)              # codes: host uint8 or CUDA uint8
    D, I = index.search(queries, k=10)       # exact top-k: the stable argsort of the
                                             # reference's distances, bit-identical
    with index.serve(k=10) as server:        # continuous batching
        req = server.submit(queries)         # non-blocking; BusyError if refused
        D, I = req.wait()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import TQError, check, lib


class BusyError(TQError):
    """The server's admission refused a request (no room in its device pool)."""


def _codes_arg(codes, cs):
    from . import _as_cai, _is_device  # the package's CUDA-array helpers (DLPack included)
    if _is_device(codes):
        codes = _as_cai(codes)
        cai = codes.__cuda_array_interface__
        total = int(np.prod(cai["shape"]))
        if total % cs:
            raise ValueError("codes size not a multiple of code_size_bytes")
        return C.c_void_p(cai["data"][0]), total // cs, 1, codes
    arr = np.ascontiguousarray(np.asarray(memoryview(codes)).view(np.uint8)).reshape(-1)
    if arr.size % cs:
        raise ValueError("codes size not a multiple of code_size_bytes")
    return C.c_void_p(arr.ctypes.data), arr.size // cs, 0, arr


class Request:
    def __init__(self, server, handle, m):
        self._server = server
        self._h = handle
        self.m = m
        self.latency_ms = None

    def done(self):
        return bool(lib().tq_request_done(self._h))

    def wait(self, timeout_ms=-1):
        k = self._server.k
        D = np.empty((self.m, k), np.float32)
        I = np.empty((self.m, k), np.int64)
        lat = C.c_double()
        check(lib().tq_request_wait(self._h, int(timeout_ms), C.c_void_p(D.ctypes.data),
                                    C.c_void_p(I.ctypes.data), C.byref(lat)))
        self.latency_ms = lat.value
        return D, I

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().tq_request_release(h)
            except Exception:
                pass
            self._h = None


class Server:
    """Continuous-batching exact top-k server over an Index.

    candidates: rows kept by the tensor-core pass for exact rescoring (0: k + 16,
    at most 32); bound_scale: multiplier on the certificate's error bound (rows
    it cannot certify are answered by an exact full pass over the codes);
    memory_budget: device bytes of the admission pool holding the queries of
    queued and in-flight requests (0: derived from the free device memory);
    queue_rows: an optional cap on queued rows (0: none beyond the pool)."""

    def __init__(self, index, k=10, max_rows=1024, slots=2, kernel_variant=-1, queue_rows=0,
                 candidates=0, bound_scale=0.0, memory_budget=0):
        self.index = index
        self.k = int(k)
        p = _capi.ServerParams(k=self.k, max_rows=int(max_rows), slots=int(slots),
                               kernel_variant=int(kernel_variant), queue_rows=int(queue_rows),
                               candidates=int(candidates), bound_scale=float(bound_scale),
                               memory_budget=int(memory_budget))
        h = C.c_void_p()
        check(lib().tq_server_create_ex(index._h, C.byref(p), C.byref(h)))
        self._h = h

    def submit(self, queries):
        space = self.index.space
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, space.dim())
        h = C.c_void_p()
        st = lib().tq_server_submit(self._h, C.c_void_p(q.ctypes.data), q.shape[0], C.byref(h))
        if st == _capi.TQ_ERR_BUSY:
            raise BusyError(st, lib().tq_last_error().decode())
        check(st)
        return Request(self, h, q.shape[0])

    def stats(self, latencies=True):
        s = _capi.ServerStats()
        n = C.c_size_t()
        check(lib().tq_server_get_stats(self._h, C.byref(s), None, 0, C.byref(n)))
        out = {f: getattr(s, f) for f, _ in _capi.ServerStats._fields_}
        if latencies and n.value:
            buf = np.empty(n.value, np.float32)
            check(lib().tq_server_get_stats(self._h, C.byref(s), C.c_void_p(buf.ctypes.data), buf.size,
                                            C.byref(n)))
            out["latencies_ms"] = buf[: n.value]
        return out

    def reset_stats(self):
        check(lib().tq_server_reset_stats(self._h))

    def tuning(self, searched=False):
        """The autotuner's choice per bucket; searched=True adds every variant's
        shape and time, and whether the choice came from the process's cache."""
        rows = (C.c_int * 16)()
        var = (C.c_int * 16)()
        ms = (C.c_float * 16)()
        n = C.c_int()
        check(lib().tq_server_tuning(self._h, rows, var, ms, 16, C.byref(n)))
        out = [{"bucket_rows": rows[i], "variant": var[i], "ms": ms[i]} for i in range(n.value)]
        if searched:
            nb, nv, cached = C.c_int(), C.c_int(), C.c_int()
            check(lib().tq_server_tuning_times(self._h, None, 0, C.byref(nb), C.byref(nv), C.byref(cached)))
            times = (C.c_float * (nb.value * nv.value))()
            check(lib().tq_server_tuning_times(self._h, times, nb.value * nv.value, C.byref(nb),
                                               C.byref(nv), C.byref(cached)))
            for i, b in enumerate(out):
                b["times_ms"] = [times[i * nv.value + v] for v in range(nv.value)]
                b["from_cache"] = bool(cached.value)
        return out


    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().tq_server_destroy(h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


LAYOUTS = {"planes": 0, "codes": 1}


class Index:
    """A corpus of codes kept in HBM for exact top-k search.

    layout "planes" (default) also keeps the codes' BF16 tensor-core operand
    planes (code_size + 6 * padded_dim + 8 bytes a code, the fastest pass);
    "codes" keeps only the codes and four floats a code, and the tensor pass
    decodes each tile of codes in shared memory (about a tenth of the memory,
    a slower pass)."""

    def __init__(self, space, codes, layout="planes"):
        self.space = space
        if layout not in LAYOUTS:
            raise ValueError(f"layout must be one of {sorted(LAYOUTS)}")
        self.layout = layout
        ptr, n, on_dev, keep = _codes_arg(codes, space.code_size_bytes())
        h = C.c_void_p()
        check(lib().tq_index_create_ex(space._h, ptr, n, on_dev, LAYOUTS[layout], C.byref(h)))
        self._h = h
        self.n = n
        self._search_server = None

    def serve(self, k=10, max_rows=1024, slots=2, kernel_variant=-1, queue_rows=0, candidates=0,
              bound_scale=0.0, memory_budget=0):
        return Server(self, k, max_rows, slots, kernel_variant, queue_rows, candidates, bound_scale,
                      memory_budget)

    def search(self, queries, k=10):
        """Exact top-k (ascending distance, ties to the smaller index) for each query row."""
        if self._search_server is None or self._search_server.k != k:
            if self._search_server is not None:
                self._search_server.close()
            self._search_server = Server(self, k, max_rows=1024, slots=1)
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, self.space.dim())
        Ds, Is = [], []
        for a in range(0, q.shape[0], 1024):
            D, I = self._search_server.submit(q[a:a + 1024]).wait()
            Ds.append(D)
            Is.append(I)
        return np.concatenate(Ds), np.concatenate(Is)

    def close(self):
        if self._search_server is not None:
            self._search_server.close()
            self._search_server = None
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().tq_index_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def variant_shapes():
    """Tile shape of each top-k kernel variant: rows per CTA, codes per tile,
    pipeline stages, K blocks per promoted chunk (0: the whole K in one
    accumulator)."""
    out = []
    v = 0
    while True:
        sh = (C.c_int * 4)()
        if lib().tq_topk_variant_shape(v, sh) != 0:
            return out
        out.append({"variant": v, "rows_per_cta": sh[0], "codes_per_tile": sh[1], "stages": sh[2],
                    "chunk_k_blocks": sh[3]})
        v += 1
