"""prepareQuery on the GPU (tq_prepare_queries_device) against the oracle,
which is pinned bit for bit to the reference build (tests/test_oracle.py):
q_rot, s_q, |q|^2 and |q| must be bit-identical (space_turbo_quant.h:439-460;
|q|^2 is the reference's sequential sum)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import turboquant as tq
from turboquant._capi import check, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,bits", [(1, 2), (3, 4), (31, 8), (100, 5), (128, 4), (768, 8),
                                      (1000, 3), (1536, 4), (4096, 6), (5000, 4)])
def test_prepare_queries_bit_exact(cuda_ok, dim, bits):
    import torch
    rng = np.random.default_rng(dim + 17 * bits)
    Q = (rng.standard_normal((37, dim)) * rng.uniform(1e-3, 1e3, (37, 1))).astype(np.float32)
    Q[0] = 0.0
    s = tq.TurboQuantSpace(dim, bits)
    D = s.padded_dim()
    Qd = torch.from_numpy(Q).cuda()
    qr = torch.empty((37, D), dtype=torch.float32, device="cuda")
    sq = torch.empty_like(qr)
    nm = torch.empty((37, 2), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    check(lib().tq_prepare_queries_device(s._h, C.c_void_p(Qd.data_ptr()), 37,
                                          C.c_void_p(qr.data_ptr()), C.c_void_p(sq.data_ptr()),
                                          C.c_void_p(nm.data_ptr()), C.c_void_p(stream)))
    torch.cuda.synchronize()
    o = O.OracleSpace(dim, bits)
    for i in range(37):
        q_rot, s_q, norms = o.prepare_query(Q[i])
        np.testing.assert_array_equal(qr[i].cpu().numpy(), q_rot)
        np.testing.assert_array_equal(sq[i].cpu().numpy(), s_q)
        np.testing.assert_array_equal(nm[i].cpu().numpy(), norms)


@pytest.mark.parametrize("dim,bits", [(3, 4), (128, 4), (768, 8), (1536, 4)])
def test_prepare_query_host_bit_exact(cuda_ok, dim, bits):
    """TurboQuantSpace.prepare_query (bindings.cpp:268-273) through the host
    entry point tq_prepare_query: the PreparedQuery's fields equal the oracle's
    bit for bit; its input checks are the reference's."""
    rng = np.random.default_rng(dim * 3 + bits)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    for q in (rng.standard_normal(dim).astype(np.float32), np.zeros(dim, np.float32)):
        pq = s.prepare_query(q)
        q_rot, s_q, norms = o.prepare_query(q)
        np.testing.assert_array_equal(pq.q_rot, q_rot)
        np.testing.assert_array_equal(pq.s_q, s_q)
        assert (np.float32(pq.q_norm_sq), np.float32(pq.q_norm)) == (norms[0], norms[1])
    with pytest.raises(ValueError, match="query: wrong length"):
        s.prepare_query(np.zeros(dim + 1, np.float32))
    with pytest.raises(ValueError):
        s.prepare_query(np.zeros(dim, np.float64))
