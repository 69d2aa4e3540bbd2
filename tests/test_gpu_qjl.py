"""Rotated coordinates and QJL-corrected symmetric distances on the GPU,
through the C ABI, against the oracle and the reference's golden vectors.

* rotated_coords_batch must be bit-identical to the reference
  (space_turbo_quant.h:411-435);
* prepare_symmetric_query must reproduce the oracle's reconstruction, signs
  and scalars bit for bit (the QJL Hadamard's butterflies are single
  roundings in the reference's stage order);
* the light / full / full-prepared distances and the 1->N prepared scan must
  agree with the reference within DIST_RTOL of the term scale; their error
  against the FP64 evaluation of the same formulas is stated.
"""
import os

import numpy as np
import pytest

import oracle as O
import turboquant as tq
from conftest import GOLDEN, dist_close, load_case, sym_term_scale

pytestmark = pytest.mark.gpu

QJL_CASES = sorted(
    tuple(int(t) for t in f[len("qjl_"):-len(".npz")].split("_"))
    for f in os.listdir(GOLDEN) if f.startswith("qjl_") and f.endswith(".npz"))
VARIANTS = (("light", "dlight"), ("full", "dfull"), ("full_prepared", "dfullp"))


def _golden(dim, bits):
    with np.load(os.path.join(GOLDEN, f"qjl_{dim}_{bits}.npz")) as z:
        return {k: z[k] for k in z.files}


def _sym(s, variant, A, B, precision="fp32"):
    return getattr(s, f"distance_m_to_n_symmetric_{variant}")(A, B, precision=precision)


@pytest.mark.parametrize("dim,bits", QJL_CASES)
def test_rotated_coords_bit_exact_vs_golden(cuda_ok, dim, bits):
    g, q = load_case(dim, bits), _golden(dim, bits)
    got = tq.TurboQuantSpace(dim, bits).rotated_coords_batch(g["X"][:8])
    np.testing.assert_array_equal(got, q["rot"])


@pytest.mark.parametrize("dim", [1, 4, 100, 768, 1536, 5000])
def test_rotated_coords_bit_exact_vs_oracle(cuda_ok, dim):
    rng = np.random.default_rng(dim)
    X = (rng.standard_normal((70, dim)) * rng.uniform(1e-3, 1e3, (70, 1))).astype(np.float32)
    X[0] = 0.0
    s = tq.TurboQuantSpace(dim, 4)
    np.testing.assert_array_equal(s.rotated_coords_batch(X),
                                  O.OracleSpace(dim, 4).rotated_coords_batch(X))


def test_rotated_coords_device_path_equals_host(cuda_ok):
    import torch
    X = np.random.default_rng(1).standard_normal((33, 300)).astype(np.float32)
    s = tq.TurboQuantSpace(300, 8)
    d = s.rotated_coords_batch(torch.from_numpy(X).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), s.rotated_coords_batch(X))


@pytest.mark.parametrize("dim,bits", QJL_CASES)
def test_symmetric_qjl_vs_golden(cuda_ok, dim, bits):
    g, q = load_case(dim, bits), _golden(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    codes = g["codes"]
    cs = s.code_size_bytes()
    ts = sym_term_scale(codes[:8], codes, cs, cs - 12)
    for variant, key in VARIANTS:
        err, ok = dist_close(_sym(s, variant, codes[:8], codes), q[key], ts)
        assert ok, f"{variant}: max rel err {err.max():.3e}"
    pq = s.prepare_symmetric_query(codes[5])
    err, ok = dist_close(s.distance_1_to_n_symmetric_full(pq, codes), q["d1full"], ts[5])
    assert ok, f"1->N full prepared: max rel err {err.max():.3e}"


@pytest.mark.parametrize("dim,bits", [(3, 2), (64, 4), (128, 8), (200, 5), (1024, 4), (768, 9),
                                      (2048, 6)])
def test_symmetric_qjl_vs_oracle_and_fp64(cuda_ok, dim, bits):
    """Several 64 x 64 tiles, ragged edges; error vs FP64 on sampled pairs."""
    rng = np.random.default_rng(dim * 3 + bits)
    X = rng.standard_normal((150, dim)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    A, B = codes[:70], codes[20:]
    cs = s.code_size_bytes()
    ts = sym_term_scale(A, B, cs, cs - 12)
    for variant in ("light", "full", "full_prepared"):
        got = _sym(s, variant, A, B)
        err, ok = dist_close(got, o.distance_m_to_n_symmetric_qjl(A, B, variant), ts)
        assert ok, f"{variant}: max rel err vs oracle {err.max():.3e}"
        pairs = rng.integers(0, [len(A), len(B)], size=(64, 2))
        d64 = np.array([o.distance_symmetric_qjl_f64(A[i], B[j], variant) for i, j in pairs])
        err64, ok64 = dist_close(got[pairs[:, 0], pairs[:, 1]], d64,
                                 ts[pairs[:, 0], pairs[:, 1]])
        assert ok64, f"{variant}: max rel err vs FP64 {err64.max():.3e}"


@pytest.mark.parametrize("dim,bits", [(3, 2), (64, 4), (128, 8), (200, 5), (1024, 4), (768, 9),
                                      (1536, 4)])
def test_symmetric_qjl_split_tf32_vs_oracle_and_fp64(cuda_ok, dim, bits):
    """The tensor-core form (two TMEM accumulators over hi/lo TF32 planes):
    two 128-row blocks and three 256-column tiles with ragged edges, every
    variant within the distance tolerance of the reference and of FP64.
    Padded dims below 64 (dim 3 here) keep the FP32 kernel."""
    rng = np.random.default_rng(dim * 7 + bits)
    X = rng.standard_normal((700, dim)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    X[3] = 0.0
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    A, B = codes[:150], codes[40:]
    cs = s.code_size_bytes()
    ts = sym_term_scale(A, B, cs, cs - 12)
    for variant in ("light", "full", "full_prepared"):
        got = _sym(s, variant, A, B, "split_tf32")
        err, ok = dist_close(got, o.distance_m_to_n_symmetric_qjl(A, B, variant), ts)
        print(f"split-TF32 {variant} {dim}/{bits}: max rel err vs oracle {err.max():.2e}")
        assert ok, f"{variant}: max rel err vs oracle {err.max():.3e}"
        pairs = rng.integers(0, [len(A), len(B)], size=(64, 2))
        d64 = np.array([o.distance_symmetric_qjl_f64(A[i], B[j], variant) for i, j in pairs])
        err64, ok64 = dist_close(got[pairs[:, 0], pairs[:, 1]], d64,
                                 ts[pairs[:, 0], pairs[:, 1]])
        assert ok64, f"{variant}: max rel err vs FP64 {err64.max():.3e}"


@pytest.mark.parametrize("dim,bits", QJL_CASES)
def test_symmetric_qjl_split_tf32_vs_golden(cuda_ok, dim, bits):
    g, q = load_case(dim, bits), _golden(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    codes = g["codes"]
    cs = s.code_size_bytes()
    ts = sym_term_scale(codes[:8], codes, cs, cs - 12)
    for variant, key in VARIANTS:
        err, ok = dist_close(_sym(s, variant, codes[:8], codes, "split_tf32"), q[key], ts)
        assert ok, f"{variant}: max rel err {err.max():.3e}"


def test_symmetric_qjl_split_tf32_device_path_equals_host(cuda_ok):
    import torch
    X = np.random.default_rng(6).standard_normal((300, 512)).astype(np.float32)
    s = tq.TurboQuantSpace(512, 4)
    codes = s.encode_batch(X)
    cd = torch.from_numpy(codes).cuda()
    for variant in ("light", "full", "full_prepared"):
        dv = _sym(s, variant, cd[:130], cd, "split_tf32")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(dv.cpu().numpy(),
                                      _sym(s, variant, codes[:130], codes, "split_tf32"))


@pytest.mark.parametrize("dim,bits", [(3, 2), (128, 4), (768, 8), (1536, 4)])
def test_prepare_symmetric_query_bit_exact(cuda_ok, dim, bits):
    X = np.random.default_rng(dim).standard_normal((4, dim)).astype(np.float32)
    s, o = tq.TurboQuantSpace(dim, bits), O.OracleSpace(dim, bits)
    codes = s.encode_batch(X)
    for c in codes:
        pq = s.prepare_symmetric_query(c)
        recon, sign, sc = o.prepare_symmetric_query(c)
        np.testing.assert_array_equal(pq.recon_q, recon)
        np.testing.assert_array_equal(pq.sign_q, sign)
        np.testing.assert_array_equal(pq.scalars, sc)


def test_prepared_paths_agree(cuda_ok):
    """distance_symmetric_full_prepared equals the 1->N scan's entry; the
    device path equals the host path; a code against itself is near zero
    (test_turboquant.py:836-846)."""
    import torch
    dim, bits = 256, 4
    X = np.random.default_rng(42).standard_normal((300, dim)).astype(np.float32)
    s = tq.TurboQuantSpace(dim, bits)
    codes = s.encode_batch(X)
    pq = s.prepare_symmetric_query(codes[7])
    d = s.distance_1_to_n_symmetric_full(pq, codes)
    assert s.distance_symmetric_full_prepared(pq, codes[11]) == d[11]
    dd = s.distance_1_to_n_symmetric_full(pq, torch.from_numpy(codes).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dd.cpu().numpy(), d)
    assert d[7] < 0.1 * float(np.sum(X[7] * X[7]))
    assert np.all(d >= 0)


def test_symmetric_qjl_device_path_equals_host(cuda_ok):
    import torch
    X = np.random.default_rng(5).standard_normal((90, 512)).astype(np.float32)
    s = tq.TurboQuantSpace(512, 8)
    codes = s.encode_batch(X)
    cd = torch.from_numpy(codes).cuda()
    for variant in ("light", "full", "full_prepared"):
        dv = _sym(s, variant, cd[:30], cd)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(dv.cpu().numpy(), _sym(s, variant, codes[:30], codes))


def test_symmetric_qjl_refuses_split_bf16(cuda_ok):
    """A BF16 pair is not accurate enough for these contractions (a code
    against itself reaches 1e-5 of the distance), so it is refused."""
    s = tq.TurboQuantSpace(256, 8)
    codes = s.encode_batch(np.random.default_rng(0).standard_normal((5, 256)).astype(np.float32))
    with pytest.raises(tq.TQError, match="SPLIT_TF32"):
        s.distance_m_to_n_symmetric_light(codes, codes, precision="split_bf16")


def test_symmetric_qjl_shapes_and_errors(cuda_ok):
    s = tq.TurboQuantSpace(64, 4)
    codes = s.encode_batch(np.random.default_rng(0).standard_normal((5, 64)).astype(np.float32))
    assert s.distance_m_to_n_symmetric_full(codes[:0], codes).shape == (0, 5)
    assert s.distance_m_to_n_symmetric_light(codes, codes[:0]).shape == (5, 0)
    with pytest.raises(ValueError, match="codes size not a multiple of code_size_bytes"):
        s.distance_m_to_n_symmetric_full(codes.reshape(-1)[:-1], codes)
    with pytest.raises(ValueError, match="codes must be uint8"):
        s.distance_m_to_n_symmetric_light(codes.astype(np.float32), codes)
    with pytest.raises(ValueError, match="code: wrong byte size"):
        s.prepare_symmetric_query(codes[0][:-1])
