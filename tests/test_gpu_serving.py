"""Serving path: device-resident index, exact top-k, continuous batching.

Top-k results are ascending by distance with ties to the smaller index, so
they must equal a stable argsort of the reference's distances, except where
two candidates' reference distances are within the distance tolerance of each
other (a near-tie may then swap).  Each request's result must be the same
whether it runs alone or batched with others.
"""
import threading

import numpy as np
import pytest

import oracle as O
import turboquant as tq
from conftest import DIST_RTOL

pytestmark = pytest.mark.gpu

DIM, BITS = 384, 4


def _mixture(rng, n, dim, centres, std=0.3):
    lab = rng.integers(0, centres.shape[0], n)
    x = centres[lab] + std * rng.standard_normal((n, dim))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


@pytest.fixture(scope="module")
def corpus(cuda_ok):
    rng = np.random.default_rng(8)
    centres = rng.standard_normal((64, DIM))
    X = _mixture(rng, 6000, DIM, centres)
    Q = _mixture(np.random.default_rng(9), 600, DIM, centres)
    space = tq.TurboQuantSpace(DIM, BITS)
    codes = space.encode_batch(X)
    ref = O.OracleSpace(DIM, BITS).distance_m_to_n(Q, codes)
    index = space.index(codes)
    yield space, codes, Q, ref, index
    index.close()


def _check_topk(D, I, ref_rows, k, qn2):
    """Valid exact top-k of the reference distances within the tolerance."""
    exact_rows = 0
    for r in range(D.shape[0]):
        ref = ref_rows[r].astype(np.float64)
        order = np.argsort(ref, kind="stable")[:k]
        tol = DIST_RTOL * max(float(np.max(np.abs(ref[order]))), qn2[r] + 1.0)
        assert np.all(np.diff(D[r]) >= 0), "not ascending"
        assert np.all(np.abs(D[r] - ref[I[r]]) <= tol), "distance differs from the reference"
        kth = ref[order[-1]]
        assert np.all(ref[I[r]] <= kth + tol), "a returned code is not in the top-k"
        mask = np.ones(ref.size, bool)
        mask[I[r]] = False
        assert np.all(ref[mask] >= kth - tol), "a better code was missed"
        exact_rows += int(np.array_equal(I[r], order))
    return exact_rows


def test_index_search_exact_topk(corpus):
    space, codes, Q, ref, index = corpus
    D, I = index.search(Q[:300], k=10)
    assert D.shape == (300, 10) and I.shape == (300, 10)
    qn2 = np.sum(Q[:300].astype(np.float64) ** 2, axis=1)
    exact = _check_topk(D, I, ref[:300], 10, qn2)
    print(f"rows whose top-10 equals the stable argsort exactly: {exact}/300")
    assert exact >= 270


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_kernel_variants_agree(corpus, variant):
    space, codes, Q, ref, index = corpus
    with index.serve(k=10, max_rows=256, slots=1, kernel_variant=variant) as sv:
        D, I = sv.submit(Q[:200]).wait()
    qn2 = np.sum(Q[:200].astype(np.float64) ** 2, axis=1)
    assert _check_topk(D, I, ref[:200], 10, qn2) >= 180


def test_same_result_alone_and_in_the_mix(corpus):
    space, codes, Q, ref, index = corpus
    sizes = [1, 7, 64, 129, 256, 3, 40, 100]
    offs = np.cumsum([0] + sizes)
    with index.serve(k=10, max_rows=512, slots=2) as sv:
        alone = [sv.submit(Q[offs[i]:offs[i + 1]]).wait() for i in range(len(sizes))]
        # the same requests submitted together from several threads, plus others
        reqs = [None] * len(sizes)
        extra = []

        def go(i):
            reqs[i] = sv.submit(Q[offs[i]:offs[i + 1]])

        ths = [threading.Thread(target=go, args=(i,)) for i in range(len(sizes))]
        for t in ths:
            t.start()
        for j in range(6):
            extra.append(sv.submit(Q[300 + 30 * j: 300 + 30 * (j + 1)]))
        for t in ths:
            t.join()
        mixed = [r.wait() for r in reqs]
        for r in extra:
            r.wait()
        st = sv.stats()
    assert st["batches"] >= 2
    for (Da, Ia), (Dm, Im) in zip(alone, mixed):
        qn2 = 1.0
        tol = DIST_RTOL * (np.abs(Da) + 2.0)
        assert np.all(np.abs(Da - Dm) <= tol)
        same = np.mean(np.all(Ia == Im, axis=1))
        assert same >= 0.95, same


def test_admission_refuses_when_queue_full(corpus):
    space, codes, Q, ref, index = corpus
    with index.serve(k=5, max_rows=256, slots=1, queue_rows=300) as sv:
        accepted, refused = [], 0
        for i in range(40):
            try:
                accepted.append(sv.submit(Q[: 100]))
            except tq.BusyError:
                refused += 1
        for r in accepted:
            D, I = r.wait()
            assert D.shape == (100, 5)
        st = sv.stats()
    assert refused > 0 and st["rejected"] == refused
    assert st["completed"] == len(accepted)


def test_autotuner_reports_each_bucket(corpus):
    space, codes, Q, ref, index = corpus
    with index.serve(k=10, max_rows=512, slots=1) as sv:
        t = sv.tuning()
    assert [b["bucket_rows"] for b in t] == [128, 256, 512]
    assert all(b["variant"] in (0, 1, 2) and b["ms"] > 0 for b in t)


def test_fewer_codes_than_k(cuda_ok):
    space = tq.TurboQuantSpace(DIM, BITS)
    rng = np.random.default_rng(1)
    codes = space.encode_batch(rng.standard_normal((5, DIM)).astype(np.float32))
    ix = space.index(codes)
    D, I = ix.search(rng.standard_normal((3, DIM)).astype(np.float32), k=8)
    assert np.all(I[:, 5:] == -1) and np.all(np.sort(I[:, :5], axis=1) == np.arange(5))
    ix.close()


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_every_column_inserts(corpus, variant):
    """Worst case for the per-row lists: the index holds the codes in order of
    descending distance to the first query, so every column of every slice
    beats that row's current k-th entry and goes through the sorted insert."""
    space, codes, Q, ref, _ = corpus
    perm = np.argsort(-ref[0].astype(np.float64), kind="stable")
    index = space.index(np.ascontiguousarray(codes[perm]))
    try:
        ref_p = ref[:64][:, perm]
        qn2 = np.sum(Q[:64].astype(np.float64) ** 2, axis=1)
        for k in (1, 10, 16):
            with index.serve(k=k, max_rows=128, slots=1, kernel_variant=variant) as sv:
                D, I = sv.submit(Q[:64]).wait()
            assert D.shape == (64, k)
            assert _check_topk(D, I, ref_p, k, qn2) >= 58
    finally:
        index.close()
