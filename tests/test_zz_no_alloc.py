"""The allocation-free scan entry point, through the C ABI.

tq_distance_1_to_n_device_noalloc serves callers that cannot allocate device
memory (a fixed memory budget reserved up front, a framework plug-in whose
enqueue must not allocate, a latency path that cannot take cudaMalloc's
synchronisation).  It keeps the prepared query in a fixed device array instead
of stream-ordered scratch.  It launches the same kernels with the same
arguments as tq_distance_1_to_n_device, only the address of the prepared query
differs, so its results must equal that entry point's bit for bit, on
consecutive calls that share the array (a stale or misplaced value in the
shared array would show as a difference).

This file is named so that pytest collects it last; it also passes on its
own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import turboquant as tq
from turboquant._capi import check, lib
from conftest import DIST_RTOL, dist_close

pytestmark = pytest.mark.gpu


def _run(fn, space, q, codes, out, stream):
    check(fn(space._h, C.c_void_p(q.data_ptr()), C.c_void_p(codes.data_ptr()), codes.shape[0],
             C.c_void_p(out.data_ptr()), C.c_void_p(stream)))


@pytest.mark.parametrize("dim,bits", [(768, 8), (128, 4)])
def test_noalloc_matches_allocating_entry_point(cuda_ok, dim, bits):
    import torch

    torch.cuda.set_device(0)
    rng = np.random.default_rng(dim + bits)
    space = tq.TurboQuantSpace(dim, bits, device=0)
    X = torch.from_numpy(rng.standard_normal((20_003, dim)).astype(np.float32)).cuda()
    codes = space.encode_batch(X)
    queries = [torch.from_numpy(rng.standard_normal(dim).astype(np.float32)).cuda() for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    L = lib()
    n = codes.shape[0]
    cs = space.code_size_bytes()
    meta = np.frombuffer(codes[:, cs - 12:cs - 8].cpu().numpy().tobytes(), np.float32).astype(np.float64)
    # two calls in a row, different queries: the second overwrites the shared scratch
    for q in queries:
        want = torch.empty(n, dtype=torch.float32, device="cuda")
        got = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
        _run(L.tq_distance_1_to_n_device, space, q, codes, want, stream)
        _run(L.tq_distance_1_to_n_device_noalloc, space, q, codes, got, stream)
        torch.cuda.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        qn2 = float(np.sum(q.cpu().numpy().astype(np.float64) ** 2))
        err, _ = dist_close(g, w, qn2 + meta ** 2, DIST_RTOL)
        assert np.array_equal(g, w), f"{int(np.sum(g != w))} distances differ, max rel {err.max():.3g}"
