"""The CPU checker (oracle/tq_oracle.c) pinned against the reference.

Golden vectors (tests/golden/, made by tests/golden/make_golden.py from the
reference compiled from its own sources) pin the restatement without the
reference present; where oracle/_ref exists (this container, or a copy of the
tree that carries it) the restatement is also checked against the reference
live on fresh seeded inputs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, GOLDEN_CASES, asym_term_scale, load_case


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_oracle_tables_match_golden(dim, bits):
    g = load_case(dim, bits)
    o = O.OracleSpace(dim, bits)
    c, b, rs, qs = o.tables()
    np.testing.assert_array_equal(c, g["centroids"])
    np.testing.assert_array_equal(b, g["boundaries"])
    np.testing.assert_array_equal(rs, g["rot_signs"])
    np.testing.assert_array_equal(qs, g["qjl_signs"])
    assert np.float32(o.scale()) == g["scale"]


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_oracle_encode_bit_exact_vs_golden(dim, bits):
    g = load_case(dim, bits)
    o = O.OracleSpace(dim, bits)
    np.testing.assert_array_equal(o.encode_batch(g["X"]), g["codes"])


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_oracle_distances_vs_golden(dim, bits):
    g = load_case(dim, bits)
    o = O.OracleSpace(dim, bits)
    codes = g["codes"]
    # asymmetric distances: the pinned build's summation order, bit for bit
    np.testing.assert_array_equal(o.distance_1_to_n(g["q"], codes).view(np.uint32),
                                  g["d1n"].view(np.uint32))
    np.testing.assert_array_equal(o.distance_m_to_n(g["Q"], codes).view(np.uint32),
                                  g["dmn"].view(np.uint32))
    # symmetric distances: the same, bit for bit
    ds = o.distance_m_to_n_symmetric(codes[:8], codes)
    np.testing.assert_array_equal(ds.view(np.uint32), g["dsym"].view(np.uint32))


def _digests():
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        return json.load(f)


def test_oracle_cfg1_digest():
    """The whole 100,000 x 128 4-bit plain-method encode, against the reference's digest."""
    X = np.random.default_rng(0).standard_normal((100_000, 128)).astype(np.float32)
    codes = O.OracleSpace(128, 4).encode_batch(X)
    assert hashlib.sha256(codes.tobytes()).hexdigest() == _digests()["cfg1_codes_sha256"]


def _cfg2_slice(rows=100_000, chunk=50_000):
    rng = np.random.default_rng(2)
    parts = []
    while rows > 0:
        k = min(chunk, rows)
        x = rng.standard_normal((k, 768)).astype(np.float32)
        n = np.linalg.norm(x, axis=1, keepdims=True)
        n[n == 0] = 1.0
        parts.append((x / n).astype(np.float32))
        rows -= k
    return np.concatenate(parts)


def test_oracle_cfg2_slice_digest():
    codes = O.OracleSpace(768, 8).encode_batch(_cfg2_slice())
    assert hashlib.sha256(codes.tobytes()).hexdigest() == _digests()["cfg2_slice_codes_sha256"]


def test_oracle_fp64_error_small():
    """The FP32 formula is within a few 1e-7 of its FP64 evaluation on typical pairs."""
    g = load_case(768, 8)
    o = O.OracleSpace(768, 8)
    ref = g["d1n"]
    f64 = np.array([o.distance_f64(g["q"], c) for c in g["codes"]])
    scale = asym_term_scale(g["q"], g["codes"], o.cs, o.cs - 12)[0]
    rel = np.abs(ref - f64) / np.maximum(np.abs(f64), scale)
    assert rel.max() < 2e-6


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("dim,bits", [(1, 2), (2, 9), (3, 4), (6, 8), (9, 5), (31, 4), (63, 6),
                                      (130, 8), (511, 4), (768, 8), (1536, 4), (3000, 7)])
def test_oracle_vs_reference_live(dim, bits):
    rng = np.random.default_rng(dim * 31 + bits)
    X = (rng.standard_normal((300, dim)) * rng.uniform(0.01, 100, (300, 1))).astype(np.float32)
    X[0] = 0
    o, r = O.OracleSpace(dim, bits), O.RefSpace(dim, bits)
    np.testing.assert_array_equal(o.encode_batch(X), r.encode_batch(X))
    q = rng.standard_normal(dim).astype(np.float32)
    for a, b in zip(o.prepare_query(q), r.prepare_query(q)):
        np.testing.assert_array_equal(a, b)
    codes = r.encode_batch(X)
    for qq in (q, np.zeros(dim, np.float32), (q * 1e-3).astype(np.float32)):
        np.testing.assert_array_equal(o.distance_1_to_n(qq, codes).view(np.uint32),
                                      r.distance_1_to_n(qq, codes).view(np.uint32))


@needs_ref
@pytest.mark.parametrize("bits", [2, 3, 4, 5, 8, 9])
def test_oracle_asym_distances_bit_exact_every_dim(bits):
    """Every padded dim 4 .. 4096: the three nibble loop shapes (D <= 16, D == 32,
    D >= 64) and the two byte shapes (D < 8, D >= 8) of the pinned build."""
    for dim in (1, 3, 5, 9, 17, 33, 64, 100, 256, 384, 768, 1024, 2048, 4096):
        rng = np.random.default_rng(dim * 7 + bits)
        X = rng.standard_normal((200, dim)).astype(np.float32)
        Q = rng.standard_normal((3, dim)).astype(np.float32)
        o, r = O.OracleSpace(dim, bits), O.RefSpace(dim, bits)
        codes = r.encode_batch(X)
        np.testing.assert_array_equal(o.distance_m_to_n(Q, codes).view(np.uint32),
                                      r.distance_m_to_n(Q, codes).view(np.uint32))


@needs_ref
@pytest.mark.parametrize("bits", [2, 3, 4, 5, 8, 9])
def test_oracle_sym_distances_bit_exact_every_dim(bits):
    """Symmetric distances in the pinned build's order, bit for bit, at every
    padded dim 4 .. 4096: the nibble shapes (<= 8 bytes, 16 bytes, blocks of 32)
    and the byte shapes (D < 8, D >= 8); zero rows and scaled rows included."""
    for dim in (1, 3, 5, 9, 17, 33, 64, 100, 256, 384, 768, 1024, 2048, 4096):
        rng = np.random.default_rng(dim * 11 + bits)
        X = (rng.standard_normal((120, dim)) * rng.uniform(1e-3, 1e3, (120, 1))).astype(np.float32)
        X[0] = 0.0
        o, r = O.OracleSpace(dim, bits), O.RefSpace(dim, bits)
        codes = r.encode_batch(X)
        np.testing.assert_array_equal(o.distance_m_to_n_symmetric(codes[:7], codes).view(np.uint32),
                                      r.distance_m_to_n_symmetric(codes[:7], codes).view(np.uint32))


@needs_ref
def test_ref_shim_equals_reference_module():
    """oracle/_ref/libtqref.so (C shim) and the reference's pybind11 module agree."""
    mod = O.import_ref_module()
    X = np.random.default_rng(5).standard_normal((500, 200)).astype(np.float32)
    a = O.RefSpace(200, 8).encode_batch(X)
    b = mod.TurboQuantSpace(200, bits_per_coord=8).encode_batch(X)
    np.testing.assert_array_equal(a, b)
