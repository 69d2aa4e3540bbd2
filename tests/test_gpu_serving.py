"""Serving path: device-resident index, exact top-k, continuous batching.

The reference has no serving loop; its top-k helpers are an argpartition +
argsort of its distances (python/tests/test_turboquant.py:270-278,
python/benchmarks/run_benchmark.py:251-255).  Here the bar is exact: every
returned row must equal the stable argsort of the reference's own distances
(the checker's, which are bit-identical to the reference build) -- the same
indices and bit-identical distances -- for k = 1, 10, 16, whether a request runs
alone or batched with others.  The certificate's fallback (a tensor-core
threshold pass whose lists are rescored, an exact scan, and a list pass for
rows the scan cannot hold) is exercised by duplicated codes and by inflated
bounds.
"""
import threading

import numpy as np
import pytest

import oracle as O
import turboquant as tq

pytestmark = pytest.mark.gpu

DIM, BITS = 384, 4


def _mixture(rng, n, dim, centres, std=0.3, chunk=50_000):
    """Rows from the 1024-centre style mixture, L2-normalised in float32."""
    parts = []
    while n > 0:
        c = min(chunk, n)
        lab = rng.integers(0, centres.shape[0], c)
        x = centres[lab] + std * rng.standard_normal((c, dim))
        parts.append((x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32))
        n -= c
    return np.concatenate(parts)


def _expect(ref_rows, k):
    """Stable argsort of the reference distances: indices and distances."""
    idx = np.argsort(ref_rows, axis=1, kind="stable")[:, :k]
    return idx, np.take_along_axis(ref_rows, idx, axis=1)


def _assert_exact(D, I, ref_rows, k):
    want_i, want_d = _expect(ref_rows, k)
    bad = np.flatnonzero(~np.all(I == want_i, axis=1))
    assert bad.size == 0, f"{bad.size} rows differ from the stable argsort, first {bad[:5]}"
    np.testing.assert_array_equal(D.view(np.uint32), want_d.astype(np.float32).view(np.uint32))


@pytest.fixture(scope="module")
def corpus(cuda_ok):
    """A config-5-shaped corpus: 384-d 4-bit codes of a 1024-centre mixture."""
    rng = np.random.default_rng(8)
    centres = rng.standard_normal((1024, DIM))
    X = _mixture(rng, 120_000, DIM, centres)
    Q = _mixture(np.random.default_rng(9), 600, DIM, centres)
    space = tq.TurboQuantSpace(DIM, BITS)
    codes = space.encode_batch(X)
    ref = O.OracleSpace(DIM, BITS).distance_m_to_n(Q, codes)
    index = space.index(codes)
    yield space, codes, X, Q, ref, index
    index.close()


@pytest.fixture(scope="module")
def index_codes(corpus):
    """The same corpus in the codes layout (B tiles decoded in shared memory)."""
    space, codes, X, Q, ref, _ = corpus
    ix = space.index(codes, layout="codes")
    yield ix
    ix.close()


@pytest.mark.parametrize("k", [1, 10, 16])
def test_index_search_is_the_stable_argsort(corpus, k):
    space, codes, X, Q, ref, index = corpus
    D, I = index.search(Q[:300], k=k)
    assert D.shape == (300, k) and I.shape == (300, k)
    _assert_exact(D, I, ref[:300], k)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6])
def test_kernel_variants_give_identical_results(corpus, variant):
    space, codes, X, Q, ref, index = corpus
    with index.serve(k=10, max_rows=256, slots=1, kernel_variant=variant) as sv:
        D, I = sv.submit(Q[:200]).wait()
        st = sv.stats()
    _assert_exact(D, I, ref[:200], 10)
    assert st["bound_violations"] == 0
    print(f"variant {variant}: {st['fallback_rows']} of 200 rows took the exact full pass")


@pytest.mark.parametrize("k", [1, 10, 16])
def test_codes_layout_is_the_stable_argsort(corpus, index_codes, k):
    space, codes, X, Q, ref, _ = corpus
    D, I = index_codes.search(Q[:300], k=k)
    _assert_exact(D, I, ref[:300], k)


@pytest.mark.parametrize("variant", [2, 4])
def test_codes_layout_variants(corpus, index_codes, variant):
    space, codes, X, Q, ref, _ = corpus
    with index_codes.serve(k=10, max_rows=256, slots=1, kernel_variant=variant) as sv:
        D, I = sv.submit(Q[:200]).wait()
        st = sv.stats()
    _assert_exact(D, I, ref[:200], 10)
    assert st["bound_violations"] == 0


def test_codes_layout_refuses_planes_only_variants(corpus, index_codes):
    # 0, 5 and 6 need planes; 1 and 3 (three stages) leave no room for a tile
    # of 268-byte codes in shared memory
    for v in (0, 1, 3, 5, 6):
        with pytest.raises(ValueError):
            index_codes.serve(k=10, max_rows=128, slots=1, kernel_variant=v)


def test_same_result_alone_and_in_the_mix(corpus):
    space, codes, X, Q, ref, index = corpus
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
    for i, ((Da, Ia), (Dm, Im)) in enumerate(zip(alone, mixed)):
        np.testing.assert_array_equal(Ia, Im)
        np.testing.assert_array_equal(Da.view(np.uint32), Dm.view(np.uint32))
        _assert_exact(Da, Ia, ref[offs[i]:offs[i + 1]], 10)


def test_duplicates_take_the_exact_fallback(corpus):
    """41 identical codes nearest to each query: the tensor pass cannot separate
    the k-th from the kc-th candidate, the certificate fails, and the exact full
    pass answers (ties broken by the smaller index)."""
    space, codes, X, Q, ref, _ = corpus
    dup = np.repeat(codes[:3], 40, axis=0)
    corp = np.ascontiguousarray(np.concatenate([codes[:20_000], dup]))
    queries = np.ascontiguousarray(np.concatenate([X[:3], Q[:13]]))
    want = O.OracleSpace(DIM, BITS).distance_m_to_n(queries, corp)
    ix = space.index(corp)
    try:
        with ix.serve(k=16, max_rows=128, slots=1) as sv:
            D, I = sv.submit(queries).wait()
            st = sv.stats()
        _assert_exact(D, I, want, 16)
        assert st["bound_violations"] == 0
        assert st["fallback_rows"] >= 3, st["fallback_rows"]
        assert st["list_pass_rows"] == 0
    finally:
        ix.close()


def test_forced_fallback_is_exact(corpus):
    """bound_scale = 1e30 makes the certificate's bound infinite: no row
    certifies, the tensor-core threshold pass would list every code, so every
    row is answered by the exact scan."""
    space, codes, X, Q, ref, _ = corpus
    ix = space.index(np.ascontiguousarray(codes[:30_000]))
    try:
        for k in (1, 10, 16):
            with ix.serve(k=k, max_rows=128, slots=1, bound_scale=1e30) as sv:
                D, I = sv.submit(Q[:50]).wait()
                st = sv.stats()
            assert st["fallback_rows"] == 50 and st["scan_pass_rows"] == 50
            assert st["list_pass_rows"] == 0
            _assert_exact(D, I, ref[:50, :30_000], k)
    finally:
        ix.close()


@pytest.mark.parametrize("layout", ["planes", "codes"])
@pytest.mark.parametrize("k", [1, 10, 16])
def test_tensor_threshold_tier_is_exact(corpus, index_codes, layout, k):
    """Inflated bounds leave many rows open: with more than four, the
    tensor-core threshold pass lists each open row's codes within e_k + eps
    and the rescoring of those lists answers them (rows whose list overflows
    go to the exact scan).  Every result is exact, and some bound of the sweep
    has rows answered from the lists."""
    space, codes, X, Q, ref, index = corpus
    ix = index if layout == "planes" else index_codes
    from_lists = 0
    for bs in (4.0, 8.0, 16.0, 32.0, 64.0):
        with ix.serve(k=k, max_rows=256, slots=1, kernel_variant=4, bound_scale=bs) as sv:
            D, I = sv.submit(Q[:256]).wait()
            st = sv.stats()
        _assert_exact(D, I, ref[:256], k)
        assert st["bound_violations"] == 0
        if st["fallback_rows"] > 4:
            from_lists += st["fallback_rows"] - st["scan_pass_rows"]
        print(f"{layout} k={k} bound x{bs}: {st['fallback_rows']} open rows, "
              f"{st['scan_pass_rows']} by the exact scan")
    assert from_lists > 0


@pytest.mark.parametrize("dim,bits", [(256, 8), (200, 3), (1000, 2), (32, 4)])
def test_forced_fallback_other_widths(cuda_ok, dim, bits):
    """The exact scan in each of its forms: term tables for nibble codes with a
    padded dim of 64 or more (200-d 3-bit, 1000-d 2-bit), the direct arithmetic
    for byte codes and for smaller nibble dims."""
    rng = np.random.default_rng(dim * 10 + bits)
    X = rng.standard_normal((7_000, dim)).astype(np.float32)
    X[::101] = 0.0
    Q = rng.standard_normal((24, dim)).astype(np.float32)
    X[3] = Q[0]
    space = tq.TurboQuantSpace(dim, bits)
    codes = space.encode_batch(X)
    want = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    ix = space.index(codes)
    try:
        with ix.serve(k=10, max_rows=128, slots=1, bound_scale=1e30) as sv:
            D, I = sv.submit(Q).wait()
            st = sv.stats()
        assert st["fallback_rows"] == 24 and st["scan_pass_rows"] == 24
        assert st["list_pass_rows"] == 0
        _assert_exact(D, I, want, 10)
    finally:
        ix.close()


def test_collection_overflow_takes_the_list_pass(corpus):
    """1,100 copies of one code at a query's smallest distance: its open row
    has more codes at or below its threshold than the exact scan collects,
    and the list pass answers it (ties by the smaller index)."""
    space, codes, X, Q, ref, _ = corpus
    dup = np.repeat(codes[5:6], 1_100, axis=0)
    corp = np.ascontiguousarray(np.concatenate([codes[:20_000], dup]))
    queries = np.ascontiguousarray(np.concatenate([X[5:6], Q[:7]]))
    want = O.OracleSpace(DIM, BITS).distance_m_to_n(queries, corp)
    ix = space.index(corp)
    try:
        with ix.serve(k=10, max_rows=128, slots=1) as sv:
            D, I = sv.submit(queries).wait()
            st = sv.stats()
        _assert_exact(D, I, want, 10)
        assert st["list_pass_rows"] >= 1, st
    finally:
        ix.close()


def test_certificate_margin_is_wide(corpus):
    """On the mixture the bound certifies (almost) every row with the default
    candidates, and no candidate ever lies outside the bound."""
    space, codes, X, Q, ref, index = corpus
    with index.serve(k=10, max_rows=512, slots=1) as sv:
        D, I = sv.submit(Q[:512]).wait()
        st = sv.stats()
    _assert_exact(D, I, ref[:512], 10)
    assert st["bound_violations"] == 0
    assert st["candidates"] == 26
    assert st["fallback_rows"] <= 5, st["fallback_rows"]


def test_admission_refuses_when_queue_full(corpus):
    space, codes, X, Q, ref, index = corpus
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
            _assert_exact(D, I, ref[:100], 5)
        st = sv.stats()
    assert refused > 0 and st["rejected"] == refused
    assert st["completed"] == len(accepted)


def test_admission_by_device_memory_budget(corpus):
    """The admission pool holds the queries of queued and in-flight requests in
    device memory: with a budget of 300 query rows, a burst of 100-row requests
    is partly refused, everything admitted completes exactly, and the pool is
    empty again afterwards."""
    space, codes, X, Q, ref, index = corpus
    row_bytes = DIM * 4
    with index.serve(k=5, max_rows=256, slots=1, memory_budget=300 * row_bytes) as sv:
        assert sv.stats()["pool_rows"] == 300
        accepted, refused = [], 0
        for i in range(40):
            try:
                accepted.append((i % 5, sv.submit(Q[100 * (i % 5): 100 * (i % 5) + 100])))
            except tq.BusyError:
                refused += 1
        for j, r in accepted:
            D, I = r.wait()
            _assert_exact(D, I, ref[100 * j: 100 * j + 100], 5)
        st = sv.stats()
    assert refused > 0 and st["rejected"] == refused
    assert st["completed"] == len(accepted)
    assert st["pool_used_rows"] == 0
    # a larger budget admits the whole burst
    with index.serve(k=5, max_rows=256, slots=1, memory_budget=4000 * row_bytes) as sv:
        rs = [sv.submit(Q[:100]) for _ in range(40)]
        for r in rs:
            r.wait()
        assert sv.stats()["rejected"] == 0


def test_budget_below_one_batch_is_refused(corpus):
    space, codes, X, Q, ref, index = corpus
    with pytest.raises(ValueError):
        index.serve(k=5, max_rows=256, slots=1, memory_budget=100 * DIM * 4)


def test_autotuner_searches_the_tile_space(corpus):
    space, codes, X, Q, ref, index = corpus
    shapes = tq.variant_shapes()
    assert len(shapes) == 7
    assert {(s["codes_per_tile"], s["stages"], s["chunk_k_blocks"]) for s in shapes} == {
        (256, 2, 8), (128, 3, 8), (128, 2, 4), (128, 3, 4), (128, 2, 8), (256, 2, 4), (256, 2, 0)}
    ix = space.index(np.ascontiguousarray(codes[:50_000]))  # an index shape not tuned before
    try:
        with ix.serve(k=10, max_rows=512, slots=1) as sv:
            t = sv.tuning(searched=True)
            D, I = sv.submit(Q[:64]).wait()
        _assert_exact(D, I, ref[:64, :50_000], 10)
        assert [b["bucket_rows"] for b in t] == [128, 256, 512]
        for b in t:
            assert not b["from_cache"]
            assert b["variant"] in range(7) and b["ms"] > 0
            assert all(x > 0 for x in b["times_ms"])
            assert b["ms"] == pytest.approx(min(b["times_ms"]))
        # the same index shape again: the process's tuning cache answers
        with ix.serve(k=10, max_rows=512, slots=1) as sv:
            t2 = sv.tuning(searched=True)
        assert all(b["from_cache"] for b in t2)
        assert [b["variant"] for b in t2] == [b["variant"] for b in t]
    finally:
        ix.close()


@pytest.mark.parametrize("layout", ["planes", "codes"])
@pytest.mark.parametrize("dim,bits", [(256, 8), (200, 3), (1000, 2), (64, 4)])
def test_other_widths_and_degenerate_codes(cuda_ok, dim, bits, layout):
    """Byte and nibble codes of other widths, with zero rows and a row equal to a
    query among them (zero gamma: the sign half left out of the tensor pass)."""
    rng = np.random.default_rng(dim + bits)
    X = rng.standard_normal((9_000, dim)).astype(np.float32)
    X[::97] = 0.0
    Q = rng.standard_normal((40, dim)).astype(np.float32)
    X[5] = Q[0]
    space = tq.TurboQuantSpace(dim, bits)
    codes = space.encode_batch(X)
    want = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    ix = space.index(codes, layout=layout)
    try:
        with ix.serve(k=10, max_rows=128, slots=1) as sv:
            D, I = sv.submit(Q).wait()
            st = sv.stats()
        _assert_exact(D, I, want, 10)
        assert st["bound_violations"] == 0
    finally:
        ix.close()


@pytest.mark.parametrize("dim,bits", [(256, 8), (200, 3), (1000, 2), (64, 4), (1536, 4)])
def test_whole_k_variant_other_widths(cuda_ok, dim, bits):
    """Variant 6 (the whole K in one accumulator) at other widths: its error
    bound grows with K (1536-d: K = 4096, 640 MMAs per accumulator), and every
    result stays the stable argsort of the reference's distances."""
    rng = np.random.default_rng(dim * 3 + bits)
    X = rng.standard_normal((6_000, dim)).astype(np.float32)
    X[::89] = 0.0
    Q = rng.standard_normal((30, dim)).astype(np.float32)
    X[7] = Q[1]
    space = tq.TurboQuantSpace(dim, bits)
    codes = space.encode_batch(X)
    want = O.OracleSpace(dim, bits).distance_m_to_n(Q, codes)
    ix = space.index(codes)
    try:
        for k in (1, 10, 16):
            with ix.serve(k=k, max_rows=128, slots=1, kernel_variant=6) as sv:
                D, I = sv.submit(Q).wait()
                st = sv.stats()
            _assert_exact(D, I, want, k)
            assert st["bound_violations"] == 0
    finally:
        ix.close()


@pytest.mark.parametrize("dim,bits", [(32, 4), (1024, 8)])
def test_codes_layout_refused_where_it_cannot_run(cuda_ok, dim, bits):
    """Padded dims below 64, and codes whose 128-code tile does not fit in
    shared memory beside two pipeline stages (1036-byte codes)."""
    space = tq.TurboQuantSpace(dim, bits)
    codes = space.encode_batch(np.ones((10, dim), np.float32))
    with pytest.raises(tq.TQError):
        space.index(codes, layout="codes")


def test_fewer_codes_than_k(cuda_ok):
    space = tq.TurboQuantSpace(DIM, BITS)
    rng = np.random.default_rng(1)
    codes = space.encode_batch(rng.standard_normal((5, DIM)).astype(np.float32))
    q = rng.standard_normal((3, DIM)).astype(np.float32)
    ix = space.index(codes)
    D, I = ix.search(q, k=8)
    ix.close()
    assert np.all(I[:, 5:] == -1) and np.all(np.isinf(D[:, 5:]))
    want = O.OracleSpace(DIM, BITS).distance_m_to_n(q, codes)
    _assert_exact(D[:, :5], I[:, :5], want, 5)


@pytest.mark.parametrize("variant", [0, 1, 5, 6])
def test_every_column_inserts(corpus, variant):
    """Worst case for the per-row lists: the index holds the codes in order of
    descending distance to the first query, so every column of every slice
    beats that row's current kc-th entry and goes through the sorted insert."""
    space, codes, X, Q, ref, _ = corpus
    perm = np.argsort(-ref[0].astype(np.float64), kind="stable")[:40_000]
    index = space.index(np.ascontiguousarray(codes[perm]))
    try:
        ref_p = np.ascontiguousarray(ref[:64][:, perm])
        for k in (1, 10, 16):
            with index.serve(k=k, max_rows=128, slots=1, kernel_variant=variant) as sv:
                D, I = sv.submit(Q[:64]).wait()
            assert D.shape == (64, k)
            _assert_exact(D, I, ref_p, k)
    finally:
        index.close()
