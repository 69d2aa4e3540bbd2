"""Parity of the CUDA path with the reference, through the C ABI.

Codes must be byte-identical (trailer floats included) to the reference's on
the same inputs; distances must agree within DIST_RTOL (conftest.py) of the
reference's, and their error against the FP64 evaluation of the same formula
is stated.  Each test runs the product path (libtqb200.so); the oracle and the
golden vectors are only the checker.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O
import turboquant as tq
from conftest import (GOLDEN, GOLDEN_CASES, asym_term_scale, dist_close, load_case,
                      sym_term_scale)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_encode_bit_exact_vs_golden(cuda_ok, dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    np.testing.assert_array_equal(s.encode_batch(g["X"]), g["codes"])


@pytest.mark.parametrize("dim,bits", [(1, 2), (2, 9), (3, 4), (4, 8), (6, 8), (9, 5), (31, 4),
                                      (32, 3), (63, 6), (64, 7), (130, 8), (256, 4), (511, 4),
                                      (768, 8), (768, 4), (1024, 9), (1536, 4), (3000, 7),
                                      (4096, 8), (8192, 4)])
def test_encode_bit_exact_vs_oracle(cuda_ok, dim, bits):
    rng = np.random.default_rng(dim * 13 + bits)
    n = 257 if dim <= 1024 else 33          # not a multiple of 3 or 4: a ragged last row group
    X = (rng.standard_normal((n, dim)) * rng.uniform(1e-3, 1e3, (n, 1))).astype(np.float32)
    X[0] = 0.0
    X[1, : max(1, dim // 2)] = 0.0
    s = tq.TurboQuantSpace(dim, bits)
    got = s.encode_batch(X)
    want = O.OracleSpace(dim, bits).encode_batch(X)
    bad = np.nonzero(np.any(got != want, axis=1))[0]
    assert bad.size == 0, f"{bad.size} rows differ, first {bad[:5]}"


def test_encode_cfg1_full_digest(cuda_ok):
    """All 100,000 codes of the 128-d 4-bit plain-method case, against the reference's digest."""
    X = np.random.default_rng(0).standard_normal((100_000, 128)).astype(np.float32)
    codes = tq.TurboQuantSpace(128, 4).encode_batch(X)
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        want = json.load(f)["cfg1_codes_sha256"]
    assert hashlib.sha256(codes.tobytes()).hexdigest() == want


def test_encode_cfg2_slice_digest(cuda_ok):
    """100,000 rows of the normalised 768-d 8-bit corpus, against the reference's digest."""
    rng = np.random.default_rng(2)
    parts = []
    for _ in range(2):
        x = rng.standard_normal((50_000, 768)).astype(np.float32)
        n = np.linalg.norm(x, axis=1, keepdims=True)
        n[n == 0] = 1.0
        parts.append((x / n).astype(np.float32))
    codes = tq.TurboQuantSpace(768, 8).encode_batch(np.concatenate(parts))
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        want = json.load(f)["cfg2_slice_codes_sha256"]
    assert hashlib.sha256(codes.tobytes()).hexdigest() == want


def test_encode_device_path_equals_host_path(cuda_ok):
    import torch
    rng = np.random.default_rng(11)
    X = rng.standard_normal((1001, 768)).astype(np.float32)
    s = tq.TurboQuantSpace(768, 8)
    host = s.encode_batch(X)
    dev = s.encode_batch(torch.from_numpy(X).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), host)
    out = torch.empty((1001, s.code_size_bytes()), dtype=torch.uint8, device="cuda")
    s.encode_batch_into(torch.from_numpy(X).cuda(), out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), host)


def test_encode_single_and_into(cuda_ok):
    g = load_case(768, 8)
    s = tq.TurboQuantSpace(768, 8)
    for i in range(5):
        np.testing.assert_array_equal(s.encode(g["X"][i]), g["codes"][i])
        buf = np.zeros(s.code_size_bytes(), np.uint8)
        s.encode_into(g["X"][i], buf)
        np.testing.assert_array_equal(buf, g["codes"][i])
    out = np.zeros(g["codes"].shape, np.uint8)
    s.encode_batch_into(g["X"], out)
    np.testing.assert_array_equal(out, g["codes"])


def test_encode_empty(cuda_ok):
    s = tq.TurboQuantSpace(128, 4)
    assert s.encode_batch(np.zeros((0, 128), np.float32)).shape == (0, 76)


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_distance_1_to_n_vs_golden(cuda_ok, dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    cs = s.code_size_bytes()
    d = s.distance_1_to_n(g["q"], g["codes"])
    err, ok = dist_close(d, g["d1n"], asym_term_scale(g["q"], g["codes"], cs, cs - 12)[0])
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_distance_m_to_n_vs_golden(cuda_ok, dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    cs = s.code_size_bytes()
    d = s.distance_m_to_n(g["Q"], g["codes"])
    assert d.shape == g["dmn"].shape
    err, ok = dist_close(d, g["dmn"], asym_term_scale(g["Q"], g["codes"], cs, cs - 12))
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_distance_symmetric_vs_golden(cuda_ok, dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    cs = s.code_size_bytes()
    A = g["codes"][:8]
    d = s.distance_m_to_n_symmetric(A, g["codes"])
    err, ok = dist_close(d, g["dsym"], sym_term_scale(A, g["codes"], cs, cs - 12))
    assert ok, err.max()


def test_single_distances_match_batch(cuda_ok):
    """distance / distance_symmetric equal the batch forms (test_turboquant.py:101-146)."""
    g = load_case(128, 4)
    s = tq.TurboQuantSpace(128, 4)
    d = s.distance_1_to_n(g["q"], g["codes"])
    for i in range(6):
        assert abs(s.distance(g["q"], g["codes"][i]) - d[i]) < 1e-4
    D = s.distance_m_to_n_symmetric(g["codes"][:3], g["codes"][:5])
    for i in range(3):
        for j in range(5):
            assert abs(s.distance_symmetric(g["codes"][i], g["codes"][j]) - D[i, j]) < 1e-4


def test_distance_cfg1_head_and_fp64_error(cuda_ok):
    """The plain-method case end to end: GPU encode, then 1->N against the
    reference's first 4096 distances; the error vs FP64 is stated."""
    X = np.random.default_rng(0).standard_normal((100_000, 128)).astype(np.float32)
    q = np.random.default_rng(1).standard_normal(128).astype(np.float32)
    s = tq.TurboQuantSpace(128, 4)
    codes = s.encode_batch(X)
    d = s.distance_1_to_n(q, codes)
    assert d.shape == (100_000,)
    with np.load(os.path.join(GOLDEN, "cfg1_d1n_head.npz")) as z:
        ref = z["d1n"]
    scale = asym_term_scale(q, codes[:4096], 76, 64)[0]
    err, ok = dist_close(d[:4096], ref, scale)
    assert ok, err.max()
    o = O.OracleSpace(128, 4)
    f64 = np.array([o.distance_f64(q, codes[i]) for i in range(0, 100_000, 97)])
    rel64 = np.abs(d[::97] - f64) / np.maximum(np.abs(f64), scale.max())
    print(f"cfg1 distance max error vs FP64: {rel64.max():.3e} (relative to term scale)")
    assert rel64.max() < 1e-5


def test_distance_cfg2_head(cuda_ok):
    rng = np.random.default_rng(2)
    x = rng.standard_normal((50_000, 768)).astype(np.float32)
    x = (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)
    q = np.random.default_rng(3).standard_normal((64, 768)).astype(np.float32)
    q = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    s = tq.TurboQuantSpace(768, 8)
    codes = s.encode_batch(x[:4096])
    d = s.distance_1_to_n(q[0], codes)
    with np.load(os.path.join(GOLDEN, "cfg2_d1n_head.npz")) as z:
        ref = z["d1n"]
    err, ok = dist_close(d, ref, asym_term_scale(q[0], codes, 1036, 1024)[0])
    assert ok, err.max()


def test_device_distances_equal_host(cuda_ok):
    import torch
    g = load_case(768, 8)
    s = tq.TurboQuantSpace(768, 8)
    codes_d = torch.from_numpy(g["codes"]).cuda()
    d1 = s.distance_1_to_n(torch.from_numpy(g["q"]).cuda(), codes_d)
    dm = s.distance_m_to_n(torch.from_numpy(g["Q"]).cuda(), codes_d)
    ds = s.distance_m_to_n_symmetric(codes_d[:8], codes_d)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d1.cpu().numpy(), s.distance_1_to_n(g["q"], g["codes"]))
    np.testing.assert_array_equal(dm.cpu().numpy(), s.distance_m_to_n(g["Q"], g["codes"]))
    np.testing.assert_array_equal(ds.cpu().numpy(),
                                  s.distance_m_to_n_symmetric(g["codes"][:8], g["codes"]))


def test_empty_and_single_row(cuda_ok):
    s = tq.TurboQuantSpace(64, 8)
    q = np.ones(64, np.float32)
    assert s.distance_1_to_n(q, np.zeros(0, np.uint8)).shape == (0,)
    codes = s.encode_batch(np.ones((1, 64), np.float32))
    assert s.distance_1_to_n(q, codes).shape == (1,)
    assert s.distance_m_to_n(np.ones((3, 64), np.float32), np.zeros(0, np.uint8)).shape == (3, 0)


# ---- M x N contractions (planes + GEMM) -----------------------------------
MTON_CASES = [(768, 4), (384, 4), (128, 4), (1024, 8), (100, 8), (1536, 4), (64, 5)]


def _oracle_mton(dim, bits, Q, codes):
    return O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)


@pytest.mark.parametrize("dim,bits", MTON_CASES)
def test_distance_m_to_n_fp32_gemm_vs_oracle(cuda_ok, dim, bits):
    """m >= 32 takes the FP32 plane GEMM path; ragged m and n (not multiples of the tiles)."""
    rng = np.random.default_rng(dim + 7 * bits)
    X = rng.standard_normal((301, dim)).astype(np.float32)
    Q = rng.standard_normal((133, dim)).astype(np.float32)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    d = s.distance_m_to_n(Q, codes)
    ref = _oracle_mton(dim, bits, Q, codes)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, asym_term_scale(Q, codes, cs, cs - 12))
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", MTON_CASES)
def test_distance_symmetric_fp32_gemm_vs_oracle(cuda_ok, dim, bits):
    rng = np.random.default_rng(dim + 11 * bits)
    s = tq.TurboQuantSpace(dim, bits)
    A = s.encode_batch(rng.standard_normal((70, dim)).astype(np.float32))
    B = s.encode_batch(rng.standard_normal((259, dim)).astype(np.float32))
    d = s.distance_m_to_n_symmetric(A, B)
    ref = O.OracleSpace(dim, bits).distance_m_to_n_symmetric(A, B)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, sym_term_scale(A, B, cs, cs - 12))
    assert ok, err.max()


def test_mton_device_gemm_equals_host(cuda_ok):
    import torch
    rng = np.random.default_rng(3)
    s = tq.TurboQuantSpace(768, 4)
    codes = s.encode_batch(rng.standard_normal((513, 768)).astype(np.float32))
    Q = rng.standard_normal((64, 768)).astype(np.float32)
    h = s.distance_m_to_n(Q, codes)
    dv = s.distance_m_to_n(torch.from_numpy(Q).cuda(), torch.from_numpy(codes).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dv.cpu().numpy(), h)


# ---- split-BF16 tcgen05 contraction ------------------------------------------
TC_CASES = [(768, 4), (1536, 4), (384, 4), (1024, 8), (100, 8), (64, 6)]


@pytest.mark.parametrize("dim,bits", TC_CASES)
def test_distance_m_to_n_split_bf16_vs_oracle(cuda_ok, dim, bits):
    rng = np.random.default_rng(dim + 3 * bits)
    X = rng.standard_normal((517, dim)).astype(np.float32)
    X = (X / np.linalg.norm(X, axis=1, keepdims=True)).astype(np.float32)
    Q = rng.standard_normal((141, dim)).astype(np.float32)
    Q = (Q / np.linalg.norm(Q, axis=1, keepdims=True)).astype(np.float32)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    d = s.distance_m_to_n(Q, codes, precision="split_bf16")
    ref = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, asym_term_scale(Q, codes, cs, cs - 12))
    print(f"split-BF16 asym {dim}/{bits}: max err {err.max():.2e}")
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", [(768, 4), (1024, 8), (64, 6)])
def test_split_bf16_exact_sign_degenerate_trailers(cuda_ok, dim, bits):
    """The split-BF16 asymmetric form divides each code's centroid half by
    g = scale * gamma and keeps its sign half exact; codes whose g is zero or
    below 1e-20 keep the plain centroid half and drop the correction term.
    Zero rows, unnormalised rows and trailers with gamma = 0 or 1e-30 agree
    with the reference within the distance tolerance."""
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
    d = s.distance_m_to_n(Q, codes, precision="split_bf16")
    ref = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    err, ok = dist_close(d, ref, asym_term_scale(Q, codes, cs, cs - 12))
    print(f"split-BF16 asym degenerate {dim}/{bits}: max err {err.max():.2e}")
    assert ok, err.max()


@pytest.mark.parametrize("dim,bits", TC_CASES)
def test_distance_symmetric_split_bf16_vs_oracle(cuda_ok, dim, bits):
    rng = np.random.default_rng(dim + 5 * bits)
    s = tq.TurboQuantSpace(dim, bits)
    A = s.encode_batch(rng.standard_normal((130, dim)).astype(np.float32))
    B = s.encode_batch(rng.standard_normal((600, dim)).astype(np.float32))
    d = s.distance_m_to_n_symmetric(A, B, precision="split_bf16")
    ref = O.OracleSpace(dim, bits).distance_m_to_n_symmetric(A, B)
    cs = s.code_size_bytes()
    err, ok = dist_close(d, ref, sym_term_scale(A, B, cs, cs - 12))
    print(f"split-BF16 sym {dim}/{bits}: max err {err.max():.2e}")
    assert ok, err.max()


def test_split_bf16_edge_shapes(cuda_ok):
    """One query row, one code, and a padded dim of 32: the asymmetric K (64)
    is a single K block with no sign-only blocks; the symmetric K (32) is not
    a whole K block and is refused with TQ_ERR_NOT_SUPPORTED."""
    from turboquant import _capi
    rng = np.random.default_rng(77)
    for dim, bits in [(32, 4), (768, 8)]:
        s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
        X = rng.standard_normal((300, dim)).astype(np.float32)
        codes = s.encode_batch(X)
        cs = s.code_size_bytes()
        for Q, C in [(X[:1], codes), (X[:130], codes[:1]), (X[:1], codes[:1])]:
            d = s.distance_m_to_n(Q, C, precision="split_bf16")
            err, ok = dist_close(d, o.distance_m_to_n(Q, C), asym_term_scale(Q, C, cs, cs - 12))
            assert d.shape == (len(Q), len(C)) and ok, (dim, d.shape, err.max())
    s = tq.TurboQuantSpace(32, 4)
    codes = s.encode_batch(rng.standard_normal((10, 32)).astype(np.float32))
    with pytest.raises(tq.TQError) as e:
        s.distance_m_to_n_symmetric(codes, codes, precision="split_bf16")
    assert e.value.status == _capi.TQ_ERR_NOT_SUPPORTED


@pytest.mark.parametrize("dim,bits", [(768, 8), (384, 4), (1536, 4), (64, 6)])
def test_distance_split_bf16_query_is_a_row(cuda_ok, dim, bits):
    """Queries equal to encoded rows: the nearest-neighbour case, where the
    terms q_rot * c mostly share a sign and the tensor core's accumulation
    drift does not average out.  Within 1e-5 of the term scale against FP64,
    on the matching pairs and on a sample of the others."""
    rng = np.random.default_rng(dim * 5 + bits)
    X = rng.standard_normal((300, dim)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    Q = X[:140].copy()
    d = s.distance_m_to_n(Q, codes, precision="split_bf16")
    pairs = [(i, i) for i in range(140)] + [tuple(p) for p in rng.integers(0, [140, 300], (200, 2))]
    ii, jj = np.array(pairs).T
    f64 = np.array([o.distance_f64(Q[i], codes[j]) for i, j in pairs])
    cs = s.code_size_bytes()
    ts = asym_term_scale(Q, codes, cs, cs - 12)[ii, jj]
    e64 = np.abs(d[ii, jj] - f64) / np.maximum(np.abs(f64), ts)
    print(f"split-BF16 asym query = row {dim}/{bits}: vs FP64 max {e64.max():.2e} "
          f"(matching pairs {e64[:140].max():.2e})")
    assert e64.max() < 1e-5, e64.max()


@pytest.mark.parametrize("dim,bits", [(768, 8), (128, 8), (1536, 4)])
@pytest.mark.parametrize("precision", ["fp32", "split_bf16"])
def test_distance_symmetric_self_pairs_vs_fp64(cuda_ok, dim, bits, precision):
    """Codes against themselves: every term of the contraction is the square
    of a centroid value, so rounding errors share a sign and add up instead of
    averaging out.  This is the worst case for the tensor-core form, and for
    the reference as well: its FP32 sum over 2048 such terms is itself 1.4e-5
    of the term scale away from FP64 here.  So the bar is 1e-5 of the term
    scale against the FP64 evaluation; against the reference, the difference
    is at most 1e-5 plus the reference's own distance from FP64."""
    rng = np.random.default_rng(dim + 11 * bits)
    X = rng.standard_normal((260, dim)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    d = s.distance_m_to_n_symmetric(codes[:130], codes, precision=precision)
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
    print(f"{precision} sym self pairs {dim}/{bits}: vs FP64 max {e64.max():.2e}; "
          f"reference vs FP64 max {r64.max():.2e}; vs reference max {eref.max():.2e}")
    assert e64.max() < 1e-5, e64.max()
    assert np.all(eref <= 1e-5 + r64), (eref - r64).max()


def test_split_bf16_error_vs_fp64(cuda_ok):
    """Error of the tensor-core form against the FP64 evaluation, 10,000 sampled pairs."""
    rng = np.random.default_rng(10)
    dim, bits = 768, 4
    X = rng.standard_normal((4096, dim)).astype(np.float32)
    X = (X / np.linalg.norm(X, axis=1, keepdims=True)).astype(np.float32)
    Q = rng.standard_normal((256, dim)).astype(np.float32)
    Q = (Q / np.linalg.norm(Q, axis=1, keepdims=True)).astype(np.float32)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    d_tc = s.distance_m_to_n(Q, codes, precision="split_bf16")
    d_32 = s.distance_m_to_n(Q, codes)
    o = O.OracleSpace(dim, bits)
    ii = rng.integers(0, 256, 10_000)
    jj = rng.integers(0, 4096, 10_000)
    f64 = np.array([o.distance_f64(Q[i], codes[j]) for i, j in zip(ii, jj)])
    scale = np.maximum(np.abs(f64), asym_term_scale(Q, codes, 524, 512)[ii, jj])
    e_tc = np.abs(d_tc[ii, jj] - f64) / scale
    e_32 = np.abs(d_32[ii, jj] - f64) / scale
    print(f"vs FP64 over 10k pairs: split-BF16 max {e_tc.max():.2e} mean {e_tc.mean():.2e}; "
          f"FP32 max {e_32.max():.2e} mean {e_32.mean():.2e}")
    assert e_tc.max() < 1e-5 and e_32.max() < 1e-5


def test_bounded_wait_reports_timeout_and_context_survives(cuda_ok):
    """A device-side wait on a barrier nothing signals gives up after its limit
    and reports TQ_ERR_TIMEOUT; the next launch on the same context works."""
    from turboquant import _capi
    st = _capi.lib().tq_selftest_bounded_wait(0, 200)
    assert st == _capi.TQ_ERR_TIMEOUT, _capi.lib().tq_last_error()
    g = load_case(128, 4)
    s = tq.TurboQuantSpace(128, 4)
    np.testing.assert_array_equal(s.encode_batch(g["X"]), g["codes"])


# ---- reference-order arithmetic (TQ_PRECISION_REFERENCE) -------------------
# The same FP32 operations in the same order as the reference's Release build
# (distSearchScalarB4 / distSearchAVX as compiled), so the distances are
# bit-identical to the reference's, not merely within the tolerance.

@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_reference_precision_bit_identical_to_golden(cuda_ok, dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    got = s.distance_m_to_n(g["Q"], g["codes"], precision="reference")
    np.testing.assert_array_equal(got.view(np.uint32), g["dmn"].view(np.uint32))


@pytest.mark.parametrize("dim,bits", [(3, 4), (17, 3), (31, 2), (33, 4), (100, 4), (384, 4),
                                      (768, 4), (1536, 4), (5, 8), (9, 5), (200, 8), (768, 8),
                                      (2048, 9), (4096, 7)])
def test_reference_precision_bit_identical_to_oracle(cuda_ok, dim, bits):
    """Every loop shape of both reference functions: nibble D <= 16, D == 32,
    D >= 64; byte D < 8, D >= 8; zero and tiny rows; the device path too."""
    import torch
    rng = np.random.default_rng(dim * 5 + bits)
    X = (rng.standard_normal((700, dim)) * rng.uniform(1e-3, 1e3, (700, 1))).astype(np.float32)
    X[0] = 0.0
    Q = rng.standard_normal((9, dim)).astype(np.float32)
    Q[0] = 0.0
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    want = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    got = s.distance_m_to_n(Q, codes, precision="reference")
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    dev = s.distance_m_to_n(torch.from_numpy(Q).cuda(), torch.from_numpy(codes).cuda(),
                            precision="reference")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy().view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_reference_precision_symmetric_bit_identical_to_golden(cuda_ok, dim, bits):
    """distBuildAVX / distBuildScalarB4 in the pinned build's order: the golden
    symmetric distances, bit for bit."""
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    codes = g["codes"]
    got = s.distance_m_to_n_symmetric(codes[:8], codes, precision="reference")
    np.testing.assert_array_equal(got.view(np.uint32), g["dsym"].view(np.uint32))


@pytest.mark.parametrize("dim,bits", [(3, 4), (17, 3), (31, 2), (33, 4), (100, 4), (384, 4),
                                      (768, 4), (1536, 4), (5, 8), (9, 5), (200, 8), (768, 8),
                                      (2048, 9), (4096, 7)])
def test_reference_precision_symmetric_bit_identical_to_oracle(cuda_ok, dim, bits):
    """Every loop shape of both symmetric reference functions (nibble: <= 8
    bytes, 16 bytes, blocks of 32; byte: D < 8, D >= 8); zero and tiny rows;
    codes against themselves; the device path too."""
    import torch
    rng = np.random.default_rng(dim * 7 + bits)
    X = (rng.standard_normal((600, dim)) * rng.uniform(1e-3, 1e3, (600, 1))).astype(np.float32)
    X[0] = 0.0
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    A = codes[:11]
    want = O.OracleSpace(dim, bits).distance_m_to_n_symmetric(A, codes)
    got = s.distance_m_to_n_symmetric(A, codes, precision="reference")
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    dev = s.distance_m_to_n_symmetric(torch.from_numpy(A).cuda(), torch.from_numpy(codes).cuda(),
                                      precision="reference")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_scan_timer_counts_launches(cuda_ok):
    """The scan kernel timer records one event pair per 1->N scan launch while on."""
    import ctypes as C
    import torch
    from turboquant._capi import check, lib
    L = lib()
    s = tq.TurboQuantSpace(256, 8)
    rng = np.random.default_rng(3)
    codes = torch.from_numpy(s.encode_batch(rng.standard_normal((50_000, 256)).astype(np.float32))).cuda()
    q = torch.from_numpy(rng.standard_normal(256).astype(np.float32)).cuda()
    out = torch.empty(50_000, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def call():
        check(L.tq_distance_1_to_n_device(s._h, C.c_void_p(q.data_ptr()), C.c_void_p(codes.data_ptr()),
                                          50_000, C.c_void_p(out.data_ptr()), C.c_void_p(st)))

    call()
    check(L.tq_space_scan_timer(s._h, 1))
    for _ in range(7):
        call()
    check(L.tq_space_scan_timer(s._h, 0))
    call()
    ms, k = C.c_double(), C.c_uint64()
    check(L.tq_space_scan_timer_read(s._h, C.byref(ms), C.byref(k)))
    assert k.value == 7 and ms.value > 0.0
    check(L.tq_space_scan_timer(s._h, 1))
    check(L.tq_space_scan_timer_read(s._h, C.byref(ms), C.byref(k)))
    assert k.value == 0 and ms.value == 0.0
