"""The CPU checker's rotated coordinates and QJL-corrected symmetric distances
pinned against the reference.

rotated_coords_batch (space_turbo_quant.h:411-435) must be bit-identical; the
light / full / full-prepared symmetric distances (:483-572, 731-945) and the
1->N full-prepared scan (:535-545) must agree within DIST_RTOL of the term
scale.  The golden vectors (tests/golden/qjl_*.npz, from the reference module
built from its own sources) pin the restatement without the reference present;
where oracle/_ref exists it is also checked live on fresh inputs.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, dist_close, load_case, sym_term_scale

QJL_CASES = sorted(
    tuple(int(t) for t in f[len("qjl_"):-len(".npz")].split("_"))
    for f in os.listdir(GOLDEN) if f.startswith("qjl_") and f.endswith(".npz"))

needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "libtqref.so")),
                               reason="reference build (oracle/_ref) not present")


def _qjl_golden(dim, bits):
    with np.load(os.path.join(GOLDEN, f"qjl_{dim}_{bits}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("dim,bits", QJL_CASES)
def test_rotated_coords_bit_exact_vs_golden(dim, bits):
    g, q = load_case(dim, bits), _qjl_golden(dim, bits)
    got = O.OracleSpace(dim, bits).rotated_coords_batch(g["X"][:8])
    np.testing.assert_array_equal(got, q["rot"])


@pytest.mark.parametrize("dim,bits", QJL_CASES)
def test_symmetric_qjl_vs_golden(dim, bits):
    g, q = load_case(dim, bits), _qjl_golden(dim, bits)
    o = O.OracleSpace(dim, bits)
    codes = g["codes"]
    cs = o.code_size_bytes()
    ts = sym_term_scale(codes[:8], codes, cs, cs - 12)
    for variant, key in (("light", "dlight"), ("full", "dfull"), ("full_prepared", "dfullp")):
        got = o.distance_m_to_n_symmetric_qjl(codes[:8], codes, variant)
        err, ok = dist_close(got, q[key], ts)
        assert ok, f"{variant}: max rel err {err.max():.3e}"
    d1 = o.distance_1_to_n_symmetric_full(o.prepare_symmetric_query(codes[5]), codes)
    err, ok = dist_close(d1, q["d1full"], ts[5])
    assert ok, f"1->N full prepared: max rel err {err.max():.3e}"


@pytest.mark.parametrize("dim,bits", [(128, 8), (768, 4)])
def test_symmetric_qjl_fp32_close_to_fp64(dim, bits):
    """The FP32 restatement is within 1e-6 of the term scale of the FP64
    evaluation of the same formulas on the same codes."""
    rng = np.random.default_rng(dim + bits)
    X = rng.standard_normal((24, dim)).astype(np.float32)
    o = O.OracleSpace(dim, bits)
    codes = o.encode_batch(X)
    cs = o.code_size_bytes()
    ts = sym_term_scale(codes[:4], codes, cs, cs - 12)
    for variant in ("light", "full", "full_prepared"):
        d32 = o.distance_m_to_n_symmetric_qjl(codes[:4], codes, variant)
        d64 = np.array([[o.distance_symmetric_qjl_f64(codes[i], codes[j], variant)
                         for j in range(len(codes))] for i in range(4)])
        err, ok = dist_close(d32, d64, ts, rtol=1e-6)
        assert ok, f"{variant}: max rel err vs FP64 {err.max():.3e}"


@needs_ref
@pytest.mark.parametrize("dim,bits", [(64, 4), (200, 8), (1024, 4), (300, 5)])
def test_qjl_vs_reference_live(dim, bits):
    R = O.import_ref_module()
    rng = np.random.default_rng(dim * 7 + bits)
    X = (rng.standard_normal((40, dim)) * rng.uniform(0.1, 10, (40, 1))).astype(np.float32)
    o, r = O.OracleSpace(dim, bits), R.TurboQuantSpace(dim, bits)
    np.testing.assert_array_equal(o.rotated_coords_batch(X), r.rotated_coords_batch(X))
    codes = r.encode_batch(X)
    cs = o.code_size_bytes()
    ts = sym_term_scale(codes[:10], codes, cs, cs - 12)
    for variant, fn in (("light", r.distance_m_to_n_symmetric_light),
                        ("full", r.distance_m_to_n_symmetric_full),
                        ("full_prepared", r.distance_m_to_n_symmetric_full_prepared)):
        err, ok = dist_close(o.distance_m_to_n_symmetric_qjl(codes[:10], codes, variant),
                             fn(codes[:10], codes), ts)
        assert ok, f"{variant}: max rel err {err.max():.3e}"
