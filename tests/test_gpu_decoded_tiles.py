"""The split-BF16 M x N distances with column tiles decoded in shared memory
(precision "split_bf16_decoded", TQ_PRECISION_SPLIT_BF16_DECODED), through
the C ABI.

The reference's distanceBatchMToN / distanceBatchMToNSymmetric
(space_turbo_quant.h:588-615) decode every code on the fly; this form does the
same per tile of 128 codes in shared memory (the centroid values as BF16 hi/lo
pairs, the QJL signs as exact +-1) and runs the three cross products on the
tensor cores, with no BF16 planes of the columns in device memory.  Distances
must agree with the reference within DIST_RTOL (conftest.py), and with the
FP64 evaluation of the same formula within 1e-5 of the term scale.
"""
import numpy as np
import pytest

import oracle as O
import turboquant as tq
from conftest import asym_term_scale, dist_close, sym_term_scale

pytestmark = pytest.mark.gpu

PREC = "split_bf16_decoded"
# (dim, bits): padded dims 64..1024, nibble and byte codes; every case's
# 128-code tile fits beside the pipeline
DEC_CASES = [(768, 4), (384, 4), (300, 8), (100, 8), (64, 6), (200, 3), (1000, 2)]


def _unit_rows(rng, n, dim):
    X = rng.standard_normal((n, dim)).astype(np.float32)
    return (X / np.linalg.norm(X, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("dim,bits", DEC_CASES)
@pytest.mark.parametrize("n", [517, 516, 128])
def test_decoded_asym_vs_oracle(cuda_ok, dim, bits, n):
    """n = 517 leaves a ragged last tile whose bytes do not end on a 16-byte
    boundary (read from a padded copy); 516 one that does (read in place);
    128 one whole tile."""
    rng = np.random.default_rng(dim + 3 * bits + n)
    X = _unit_rows(rng, n, dim)
    Q = _unit_rows(rng, 141, dim)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    d = s.distance_m_to_n(Q, codes, precision=PREC)
    ref = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, asym_term_scale(Q, codes, cs, cs - 12))
    print(f"decoded asym {dim}/{bits} n={n}: max err {err.max():.2e}")
    assert d.shape == (141, n) and ok, err.max()


@pytest.mark.parametrize("dim,bits", DEC_CASES)
def test_decoded_sym_vs_oracle(cuda_ok, dim, bits):
    rng = np.random.default_rng(dim + 5 * bits)
    s = tq.TurboQuantSpace(dim, bits)
    A = s.encode_batch(rng.standard_normal((130, dim)).astype(np.float32))
    B = s.encode_batch(rng.standard_normal((601, dim)).astype(np.float32))
    d = s.distance_m_to_n_symmetric(A, B, precision=PREC)
    ref = O.OracleSpace(dim, bits).distance_m_to_n_symmetric(A, B)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, sym_term_scale(A, B, cs, cs - 12))
    print(f"decoded sym {dim}/{bits}: max err {err.max():.2e}")
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", [(768, 4), (300, 8), (64, 6)])
def test_decoded_degenerate_trailers(cuda_ok, dim, bits):
    """Codes whose scale * gamma is zero or below 1e-20 take the plain
    centroid factor (sigma) and a zero sign-half factor, as the planes form;
    zero rows and zero queries included."""
    rng = np.random.default_rng(dim + 7 * bits)
    X = (rng.standard_normal((300, dim)) * rng.uniform(1e-3, 1e3, (300, 1))).astype(np.float32)
    X[0] = 0.0
    Q = rng.standard_normal((130, dim)).astype(np.float32)
    Q[1] = 0.0
    s = tq.TurboQuantSpace(dim, bits)
    cs = s.code_size_bytes()
    codes = s.encode_batch(X)
    gam = codes[:, cs - 8:cs - 4].copy().view(np.float32)
    gam[3:40] = 0.0
    gam[40:60] = 1e-30
    codes[:, cs - 8:cs - 4] = gam.view(np.uint8)
    d = s.distance_m_to_n(Q, codes, precision=PREC)
    ref = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    err, ok = dist_close(d, ref, asym_term_scale(Q, codes, cs, cs - 12))
    print(f"decoded asym degenerate {dim}/{bits}: max err {err.max():.2e}")
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", [(768, 4), (384, 4), (300, 8), (64, 6)])
def test_decoded_query_is_a_row_vs_fp64(cuda_ok, dim, bits):
    """The nearest-neighbour case (a query equal to an encoded row), where the
    terms share a sign and the accumulation drift does not average out."""
    rng = np.random.default_rng(dim * 5 + bits)
    X = _unit_rows(rng, 300, dim)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    Q = X[:140].copy()
    d = s.distance_m_to_n(Q, codes, precision=PREC)
    pairs = [(i, i) for i in range(140)] + [tuple(p) for p in rng.integers(0, [140, 300], (200, 2))]
    ii, jj = np.array(pairs).T
    f64 = np.array([o.distance_f64(Q[i], codes[j]) for i, j in pairs])
    cs = s.code_size_bytes()
    ts = asym_term_scale(Q, codes, cs, cs - 12)[ii, jj]
    e64 = np.abs(d[ii, jj] - f64) / np.maximum(np.abs(f64), ts)
    print(f"decoded asym query = row {dim}/{bits}: vs FP64 max {e64.max():.2e} "
          f"(matching pairs {e64[:140].max():.2e})")
    assert e64.max() < 1e-5, e64.max()


@pytest.mark.parametrize("dim,bits", [(768, 4), (128, 8), (300, 8)])
def test_decoded_sym_self_pairs_vs_fp64(cuda_ok, dim, bits):
    """Codes against themselves (squares of centroid values): within 1e-5 of
    the term scale against FP64, and within 1e-5 plus the reference's own
    distance from FP64 against the reference."""
    rng = np.random.default_rng(dim + 11 * bits)
    X = _unit_rows(rng, 260, dim)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    d = s.distance_m_to_n_symmetric(codes[:130], codes, precision=PREC)
    ref = o.distance_m_to_n_symmetric(codes[:130], codes)
    pairs = [(i, i) for i in range(130)] + [tuple(p) for p in rng.integers(0, [130, 260], (200, 2))]
    ii, jj = np.array(pairs).T
    f64 = np.array([o.distance_symmetric_f64(codes[i], codes[j]) for i, j in pairs])
    cs = s.code_size_bytes()
    ts = sym_term_scale(codes[:130], codes, cs, cs - 12)[ii, jj]
    den = np.maximum(np.abs(f64), ts)
    e64 = np.abs(d[ii, jj] - f64) / den
    r64 = np.abs(ref[ii, jj] - f64) / den
    eref = np.abs(d[ii, jj] - ref[ii, jj]) / den
    print(f"decoded sym self pairs {dim}/{bits}: vs FP64 max {e64.max():.2e}; "
          f"reference vs FP64 max {r64.max():.2e}")
    assert e64.max() < 1e-5, e64.max()
    assert np.all(eref <= 1e-5 + r64), (eref - r64).max()


def test_decoded_error_vs_fp64_and_planes(cuda_ok):
    """768-d 4-bit (the dense batch's shapes, fewer rows): error against the
    FP64 evaluation over 10,000 sampled pairs, beside the planes form."""
    rng = np.random.default_rng(10)
    dim, bits = 768, 4
    X = _unit_rows(rng, 4096, dim)
    Q = _unit_rows(rng, 256, dim)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    d_dec = s.distance_m_to_n(Q, codes, precision=PREC)
    d_pl = s.distance_m_to_n(Q, codes, precision="split_bf16")
    o = O.OracleSpace(dim, bits)
    ii = rng.integers(0, 256, 10_000)
    jj = rng.integers(0, 4096, 10_000)
    f64 = np.array([o.distance_f64(Q[i], codes[j]) for i, j in zip(ii, jj)])
    scale = np.maximum(np.abs(f64), asym_term_scale(Q, codes, 524, 512)[ii, jj])
    e_dec = np.abs(d_dec[ii, jj] - f64) / scale
    e_pl = np.abs(d_pl[ii, jj] - f64) / scale
    print(f"vs FP64 over 10k pairs: decoded max {e_dec.max():.2e} mean {e_dec.mean():.2e}; "
          f"planes max {e_pl.max():.2e} mean {e_pl.mean():.2e}")
    assert e_dec.max() < 1e-5 and e_pl.max() < 1e-5


def test_decoded_device_path_equals_host(cuda_ok):
    """Device buffers (torch CUDA tensors) give the host path's distances bit
    for bit: the same kernels on the same bytes."""
    import torch

    rng = np.random.default_rng(21)
    dim, bits = 384, 4
    s = tq.TurboQuantSpace(dim, bits)
    X = _unit_rows(rng, 1003, dim)
    Q = _unit_rows(rng, 70, dim)
    codes = s.encode_batch(X)
    h = s.distance_m_to_n(Q, codes, precision=PREC)
    dv = s.distance_m_to_n(torch.from_numpy(Q).cuda(), torch.from_numpy(codes).cuda(), precision=PREC)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dv.cpu().numpy(), h)
    hs = s.distance_m_to_n_symmetric(codes[:65], codes, precision=PREC)
    ds = s.distance_m_to_n_symmetric(torch.from_numpy(codes[:65]).cuda(), torch.from_numpy(codes).cuda(),
                                     precision=PREC)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ds.cpu().numpy(), hs)


def test_decoded_refusals(cuda_ok):
    """Shapes the decoded form does not take are refused with
    TQ_ERR_NOT_SUPPORTED, never computed another way: a padded dim below 64,
    a code tile too large for shared memory (1024-d byte codes, 1,036 B) and
    device codes that are not 16-byte aligned."""
    import torch
    from turboquant import _capi

    rng = np.random.default_rng(5)
    for dim, bits in [(32, 4), (1024, 8)]:
        s = tq.TurboQuantSpace(dim, bits)
        X = rng.standard_normal((10, dim)).astype(np.float32)
        codes = s.encode_batch(X)
        with pytest.raises(tq.TQError) as e:
            s.distance_m_to_n(X, codes, precision=PREC)
        assert e.value.status == _capi.TQ_ERR_NOT_SUPPORTED
        with pytest.raises(tq.TQError) as e:
            s.distance_m_to_n_symmetric(codes, codes, precision=PREC)
        assert e.value.status == _capi.TQ_ERR_NOT_SUPPORTED
    s = tq.TurboQuantSpace(128, 4)
    cs = s.code_size_bytes()
    X = rng.standard_normal((300, 128)).astype(np.float32)
    codes = s.encode_batch(X)
    raw = torch.zeros(300 * cs + 16, dtype=torch.uint8, device="cuda")
    view = raw[4:4 + 300 * cs].view(300, cs)  # 4-byte aligned, not 16
    view.copy_(torch.from_numpy(codes).cuda())
    with pytest.raises(tq.TQError) as e:
        s.distance_m_to_n(torch.from_numpy(X[:5]).cuda(), view, precision=PREC)
    assert e.value.status == _capi.TQ_ERR_NOT_SUPPORTED
