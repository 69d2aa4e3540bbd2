"""Generate the golden vectors under tests/golden/ from the reference itself.

Run in a container that has the reference sources: it builds the reference
from them (oracle/Makefile, target ``ref``) and records, per (dim, bits) case,
the reference's own outputs on seeded inputs:

* ``case_<dim>_<bits>.npz``: X, codes (encode_batch), q + d1n (distance_1_to_n),
  Q + dmn (distance_m_to_n), dsym (distance_m_to_n_symmetric of the first rows
  against all rows), the tables (centroids, boundaries, signs) and scale;
* ``digests.json``: SHA-256 of the reference codes of larger seeded inputs
  (the full 100,000 x 128 config of the reference's small plain-method case and
  a 100,000-row slice of the 768-d 8-bit corpus), with the generating recipe.

The inputs follow the reference's own test pattern
(``np.random.default_rng(seed).standard_normal(shape).astype(np.float32)``,
python/tests/test_turboquant.py:17-19) and its benchmark's row normalisation
(python/benchmarks/run_benchmark.py:229-232).

* ``qjl_<dim>_<bits>.npz`` (``make_golden.py qjl``): rotated_coords_batch and
  the QJL-corrected symmetric distances of the reference module on the same
  inputs.

Usage:  python tests/golden/make_golden.py [qjl]
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

# (dim, bits): the benchmark workloads' shapes (128-d and 384-d 4-bit, 768-d 8- and
# 4-bit, 1536-d 4-bit) plus the edge cases of the layout
# (nibble vs byte, padding, dim < 4, 9-bit overflow of the unit byte).
CASES = [
    (128, 4), (768, 8), (768, 4), (1536, 4), (384, 4),
    (1, 2), (3, 3), (5, 2), (7, 4), (17, 5), (33, 6), (64, 7), (100, 9), (200, 8),
    (255, 4), (1000, 3), (2048, 8), (4096, 4),
]


def l2_normalize(x):
    """run_benchmark.py:229-232"""
    n = np.linalg.norm(x, axis=1, keepdims=True)
    n[n == 0] = 1.0
    return (x / n).astype(np.float32)


def case_inputs(dim, bits, n=32, m=4):
    rng = np.random.default_rng(1000 * dim + bits)
    X = rng.standard_normal((n, dim)).astype(np.float32)
    X[0] = 0.0                       # zero row: inv_norm = 0 path
    X[1] *= np.float32(1e-12)        # tiny norm
    X[2] *= np.float32(1e15)         # huge norm
    X[3, ::3] = 0.0                  # exact zeros inside a row
    X[4] = np.abs(X[4])              # one-signed row
    Q = rng.standard_normal((m, dim)).astype(np.float32)
    q = rng.standard_normal(dim).astype(np.float32)
    return X, q, Q


def digest(b: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()


def cfg1_inputs():
    """dim 128, b4: X 100,000 x 128 N(0,1) seed 0 (not normalised); q seed 1."""
    X = np.random.default_rng(0).standard_normal((100_000, 128)).astype(np.float32)
    q = np.random.default_rng(1).standard_normal(128).astype(np.float32)
    return X, q


def cfg2_slice(rows=100_000, chunk=50_000):
    """dim 768, b8: rows of the seed-2 N(0,1) corpus, L2-normalised per row,
    drawn in chunks from one generator."""
    rng = np.random.default_rng(2)
    parts = []
    left = rows
    while left > 0:
        k = min(chunk, left)
        parts.append(l2_normalize(rng.standard_normal((k, 768)).astype(np.float32)))
        left -= k
    return np.concatenate(parts)


def main():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "liboracle.so"], check=True)
    for dim, bits in CASES:
        r = O.RefSpace(dim, bits)
        X, q, Q = case_inputs(dim, bits)
        codes = r.encode_batch(X)
        d1n = r.distance_1_to_n(q, codes)
        dmn = r.distance_m_to_n(Q, codes)
        dsym = r.distance_m_to_n_symmetric(codes[:8], codes)
        c, b, rs, qs = r.tables()
        np.savez_compressed(
            os.path.join(HERE, f"case_{dim}_{bits}.npz"), dim=dim, bits=bits, X=X, codes=codes,
            q=q, d1n=d1n, Q=Q, dmn=dmn, dsym=dsym, centroids=c, boundaries=b, rot_signs=rs,
            qjl_signs=qs, scale=np.float32(r.scale()))
        print("case", dim, bits, codes.shape)

    X1, q1 = cfg1_inputs()
    r1 = O.RefSpace(128, 4)
    c1 = r1.encode_batch(X1)
    d1 = r1.distance_1_to_n(q1, c1)
    np.savez_compressed(os.path.join(HERE, "cfg1_d1n_head.npz"), d1n=d1[:4096])
    X2 = cfg2_slice()
    r2 = O.RefSpace(768, 8)
    c2 = r2.encode_batch(X2)
    q2 = l2_normalize(np.random.default_rng(3).standard_normal((64, 768)).astype(np.float32))
    d2 = r2.distance_1_to_n(q2[0], c2[:4096])
    np.savez_compressed(os.path.join(HERE, "cfg2_d1n_head.npz"), d1n=d2)
    meta = {
        "generator": "tests/golden/make_golden.py",
        "reference_build": "oracle/Makefile target ref: g++ -O3 -ffast-math -fno-finite-math-only "
                           "-march=x86-64-v3 -std=c++17 -DNDEBUG -fopenmp",
        "cfg1_codes_sha256": digest(c1),
        "cfg1_recipe": "default_rng(0).standard_normal((100000,128)).astype(float32); dim 128 bits 4",
        "cfg2_slice_codes_sha256": digest(c2),
        "cfg2_slice_recipe": "default_rng(2) chunks of 50000 x 768 standard_normal -> float32 -> "
                             "l2 normalise per row; first 100000 rows; dim 768 bits 8",
    }
    with open(os.path.join(HERE, "digests.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta, indent=1))


# (dim, bits) cases of the rotated-coordinate diagnostic and the QJL-corrected
# symmetric distances (reference module methods rotated_coords_batch,
# distance_m_to_n_symmetric_{light,full,full_prepared},
# prepare_symmetric_query + distance_1_to_n_symmetric_full).
QJL_CASES = [(128, 4), (768, 8), (1536, 4), (384, 4), (7, 4), (33, 6), (100, 9), (1000, 3)]


def qjl_main():
    """``qjl_<dim>_<bits>.npz``: the reference module's outputs on the inputs
    and codes of ``case_<dim>_<bits>.npz`` (the first 8 rows against all 32)."""
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    R = O.import_ref_module()
    for dim, bits in QJL_CASES:
        r = R.TurboQuantSpace(dim, bits)
        X, _, _ = case_inputs(dim, bits)
        codes = r.encode_batch(X)
        prev = np.load(os.path.join(HERE, f"case_{dim}_{bits}.npz"))["codes"]
        assert np.array_equal(prev, codes), "inputs differ from case_<dim>_<bits>.npz"
        np.savez_compressed(
            os.path.join(HERE, f"qjl_{dim}_{bits}.npz"),
            rot=r.rotated_coords_batch(X[:8]),
            dlight=r.distance_m_to_n_symmetric_light(codes[:8], codes),
            dfull=r.distance_m_to_n_symmetric_full(codes[:8], codes),
            dfullp=r.distance_m_to_n_symmetric_full_prepared(codes[:8], codes),
            d1full=r.distance_1_to_n_symmetric_full(r.prepare_symmetric_query(codes[5]), codes))
        print("qjl", dim, bits)


if __name__ == "__main__":
    if sys.argv[1:] == ["qjl"]:
        qjl_main()
    else:
        main()
