"""Shared test setup.

* registers the ``gpu`` marker (tests that need a B200; run with ``-m gpu``);
* puts the product package (turboquant-space_b200/python) and the CPU checker
  (oracle/) on sys.path;
* builds liboracle.so (the plain-C restatement) on demand.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "turboquant-space_b200", "python")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")


GOLDEN_CASES = sorted(
    tuple(int(t) for t in f[len("case_"):-len(".npz")].split("_"))
    for f in os.listdir(GOLDEN) if f.startswith("case_") and f.endswith(".npz"))


def load_case(dim, bits):
    with np.load(os.path.join(GOLDEN, f"case_{dim}_{bits}.npz")) as z:
        return {k: z[k] for k in z.files}


# Distance tolerance.  The reference computes d = |q|^2 + |x|^2 - 2<q,x>_est
# in FP32; for near-duplicate pairs the subtraction cancels and any change of
# summation order moves d by a few ulps of the *terms*, not of d.  So the bar
# is 1e-5 relative to max(|d_ref|, |q|^2 + |x|^2): plain relative error for
# typical pairs, the term scale for cancelling ones.
DIST_RTOL = 1e-5


def dist_close(got, ref, term_scale, rtol=DIST_RTOL):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    denom = np.maximum(np.abs(ref), np.asarray(term_scale, dtype=np.float64))
    denom = np.maximum(denom, 1e-30)
    err = np.abs(got - ref) / denom
    return err, bool(np.all(err <= rtol))


def asym_term_scale(Q, codes, cs, pb):
    """|q|^2 + |x|^2 per (query, code) pair from the FP32 inputs/trailers."""
    Q = np.atleast_2d(np.asarray(Q, np.float32)).astype(np.float64)
    qn2 = np.sum(Q * Q, axis=1)
    meta = np.frombuffer(np.ascontiguousarray(codes).reshape(-1, cs)[:, pb:pb + 12].tobytes(),
                         np.float32).reshape(-1, 3)
    xn2 = meta[:, 0].astype(np.float64) ** 2
    return qn2[:, None] + xn2[None, :]


def sym_term_scale(A, B, cs, pb):
    ma = np.frombuffer(np.ascontiguousarray(A).reshape(-1, cs)[:, pb:pb + 12].tobytes(),
                       np.float32).reshape(-1, 3)
    mb = np.frombuffer(np.ascontiguousarray(B).reshape(-1, cs)[:, pb:pb + 12].tobytes(),
                       np.float32).reshape(-1, 3)
    return ma[:, 0].astype(np.float64)[:, None] ** 2 + mb[:, 0].astype(np.float64)[None, :] ** 2


@pytest.fixture(scope="session")
def cuda_ok():
    """The GPU tests' precondition: torch sees a CUDA device of compute capability 10.x."""
    import torch
    assert torch.cuda.is_available(), "GPU test without a CUDA device"
    major, _ = torch.cuda.get_device_capability(0)
    assert major == 10, f"expected an sm_100 device, got sm_{major}x"
    return True
