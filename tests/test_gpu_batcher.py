"""Uneven batches through the captured-graph batcher: every row equals the plain batch search of
that query with its own k and ef (bit-exact), for batches of changing size replayed through the
same graph; the autotuner keeps a plan that gives the same results."""

import numpy as np
import pytest

from conftest import integer_matrix


@pytest.fixture(scope="module")
def graph(gpu):
    base = integer_matrix(3000, 24, seed=31)
    ix = gpu.HnswIndex(24, "l2", M=12, ef_construction=80)
    ix.add(base, num_threads=0)
    return ix


def expected(ix, q, k, ef, width, **opts):
    ids = np.full((len(q), width), 0xFFFFFFFF, np.uint32)
    d = np.full((len(q), width), np.inf, np.float32)
    c = np.zeros(len(q), np.uint32)
    for i in range(len(q)):
        a, b, n = ix.search_batch(q[i:i + 1], int(k[i]), int(ef[i]), **opts)
        ids[i, :k[i]], d[i, :k[i]], c[i] = a[0], b[0], n[0]
    return ids, d, c


def check(ix, bt, q, k, ef, width, **opts):
    ids, d, c = bt.run(q, k, ef)
    wi, wd, wc = expected(ix, q, k, ef, width, **opts)
    np.testing.assert_array_equal(c, wc)
    for i in range(len(q)):
        np.testing.assert_array_equal(ids[i, :k[i]], wi[i, :k[i]])
        np.testing.assert_array_equal(d[i, :k[i]], wd[i, :k[i]])


@pytest.mark.gpu
def test_uneven_batches_replay_one_graph(gpu, graph):
    bt = gpu.Batcher(graph, max_queries=300, max_k=20, max_ef=128)
    g = np.random.default_rng(5)
    for nq in (300, 1, 77, 0, 256, 13):
        q = integer_matrix(nq, 24, seed=100 + nq)
        k = g.integers(1, 21, size=nq).astype(np.uint32)
        ef = g.integers(1, 129, size=nq).astype(np.uint32)
        if nq == 0:
            ids, d, c = bt.run(q, k, ef)
            assert ids.shape == (0, 20) and len(c) == 0
            continue
        check(graph, bt, q, k, ef, 20)


@pytest.mark.gpu
def test_bf16_batcher_matches_the_bf16_search(gpu, graph):
    bt = gpu.Batcher(graph, max_queries=64, max_k=10, max_ef=64, precision="bf16")
    q = integer_matrix(64, 24, seed=7)
    k = np.array([1, 5, 10, 3] * 16, np.uint32)
    ef = np.where(np.arange(64) % 2 == 0, 16, 64).astype(np.uint32)
    # Each query's FP32 re-rank covers its best 4 * k, as the batch search's default.
    check(graph, bt, q, k, ef, 10, precision="bf16")


@pytest.mark.gpu
def test_ef_classes_split_and_rejoin_in_batch_order(gpu, graph):
    # max_ef 600 gives classes <= 64, <= 256 and <= 600; ef >= n runs exhaustively.
    bt = gpu.Batcher(graph, max_queries=120, max_k=12, max_ef=600)
    q = integer_matrix(120, 24, seed=17)
    g = np.random.default_rng(8)
    k = g.integers(1, 13, size=120).astype(np.uint32)
    ef = g.choice([5, 40, 64, 65, 200, 256, 257, 600], size=120).astype(np.uint32)
    check(graph, bt, q, k, ef, 12)


@pytest.mark.gpu
def test_autotune_keeps_results(gpu, graph):
    bt = gpu.Batcher(graph, max_queries=200, max_k=10, max_ef=64)
    q = integer_matrix(200, 24, seed=9)
    k = np.full(200, 10, np.uint32)
    ef = np.full(200, 48, np.uint32)
    before = bt.run(q, k, ef)
    timings = bt.autotune(q, k, ef)
    assert len(timings) >= 3 and all(t["ms"] > 0 for t in timings)
    assert {t["ef_class"] for t in timings} == {64}
    after = bt.run(q, k, ef)
    for x, y in zip(before, after):
        np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
def test_autotune_bf16_keeps_block_limit_and_results(gpu, graph):
    """BF16 kernels of capacity <= 64 run blocks of at most 4 warps (96 registers a thread):
    the autotuner tries only those, and its plan gives the same rows."""
    bt = gpu.Batcher(graph, max_queries=200, max_k=10, max_ef=64, precision="bf16")
    q = integer_matrix(200, 24, seed=19)
    k = np.full(200, 10, np.uint32)
    ef = np.full(200, 40, np.uint32)
    before = bt.run(q, k, ef)
    timings = bt.autotune(q, k, ef)
    assert timings and max(t["warps_per_block"] for t in timings) == 4
    after = bt.run(q, k, ef)
    for x, y in zip(before, after):
        np.testing.assert_array_equal(x, y)


@pytest.mark.gpu
def test_batcher_rejects_what_does_not_fit(gpu, graph):
    bt = gpu.Batcher(graph, max_queries=8, max_k=5, max_ef=32)
    q = integer_matrix(9, 24, seed=3)
    with pytest.raises(ValueError):
        bt.run(q, 5, 32)
    with pytest.raises(ValueError):
        bt.run(q[:4], 6, 32)
    with pytest.raises(ValueError):
        bt.run(q[:4], 5, 33)
    bad = q[:2].copy()
    bad[1, 3] = np.nan
    with pytest.raises(ValueError):
        bt.run(bad, 5, 16)
    ids, _, c = bt.run(q[:2], 5, 16)  # still usable after an error
    assert list(c) == [5, 5]


@pytest.mark.gpu
def test_batches_in_flight_on_several_batchers(gpu, graph):
    """submit / wait on two batchers with both batches in flight give the same rows as run."""
    a = gpu.Batcher(graph, max_queries=100, max_k=10, max_ef=200)
    b = gpu.Batcher(graph, max_queries=100, max_k=10, max_ef=200)
    g = np.random.default_rng(12)
    qa, qb = integer_matrix(100, 24, seed=41), integer_matrix(60, 24, seed=42)
    ka, kb = g.integers(1, 11, 100).astype(np.uint32), g.integers(1, 11, 60).astype(np.uint32)
    ea, eb = g.integers(1, 201, 100).astype(np.uint32), g.integers(1, 201, 60).astype(np.uint32)
    a.submit(qa, ka, ea)
    b.submit(qb, kb, eb)
    with pytest.raises(ValueError):
        a.submit(qa, ka, ea)  # one batch in flight per batcher
    got_b, got_a = b.wait(), a.wait()
    for got, (q, k, e) in ((got_a, (qa, ka, ea)), (got_b, (qb, kb, eb))):
        want = a.run(q, k, e)
        for x, y in zip(got, want):
            np.testing.assert_array_equal(x, y)
