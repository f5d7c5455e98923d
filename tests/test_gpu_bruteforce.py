"""GPU exact brute force through the C ABI against the reference's BruteForceIndex: known
answers, and bit-exact ids and distances for every metric."""

from pathlib import Path

import numpy as np
import pytest

from conftest import integer_matrix, uniform_matrix

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
METHODS = ["exact", "tensor_core"]


def method_available(gpu, method):
    if method == "exact":
        return True
    bf = gpu.BruteForceIndex(4)
    bf.add(uniform_matrix(64, 4, 1))
    try:
        bf.search_batch(uniform_matrix(2, 4, 2), 2, method=method)
        return True
    except RuntimeError:
        return False


@pytest.mark.parametrize("method", METHODS)
def test_known_answers(gpu, method):
    if not method_available(gpu, method):
        pytest.skip("tensor-core brute force not available")
    line = gpu.BruteForceIndex(1)
    line.add(np.array([[10.0], [0.0], [7.0], [3.0], [-2.0]], np.float32))
    assert line.search([2.0], 3) == [(1.0, 3), (4.0, 1), (16.0, 4)]
    two = gpu.BruteForceIndex(1)
    two.add(np.array([[5.0], [1.0]], np.float32))
    assert two.search([0.0], 10) == [(1.0, 1), (25.0, 0)]
    ties = gpu.BruteForceIndex(1)
    ties.add(np.array([[4.0], [-4.0], [4.0], [9.0], [-4.0]], np.float32))
    assert ties.search([0.0], 4) == [(16.0, 0), (16.0, 1), (16.0, 2), (16.0, 4)]
    assert ties.search([0.0], 2) == [(16.0, 0), (16.0, 1)]
    ip = gpu.BruteForceIndex(2, "ip")
    ip.add(np.array([[1, 0], [0, 2], [3, 3]], np.float32))
    assert ip.search([1.0, 1.0], 3) == [(-5.0, 2), (-1.0, 1), (0.0, 0)]
    cos = gpu.BruteForceIndex(2, "cosine")
    cos.add(np.array([[10, 0], [0, 0.5], [-3, 0]], np.float32))
    assert cos.search([2.0, 0.0], 3) == [(0.0, 0), (1.0, 1), (2.0, 2)]
    assert gpu.BruteForceIndex(3).search([1.0, 2.0, 3.0], 5) == []


def test_golden_bruteforce(gpu):
    g = np.load(GOLDEN / "kat_results.npz")
    bf = gpu.BruteForceIndex(16)
    bf.add(integer_matrix(1000, 16, 1))
    ids, d, c = bf.search_batch(integer_matrix(200, 16, 2), 10)
    np.testing.assert_array_equal(ids, g["bf_ids"])
    np.testing.assert_array_equal(d, g["bf_dists"])


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [16, 24, 100, 128])
def test_exact_equals_reference(gpu, orc, metric, dim):
    base = uniform_matrix(3000, dim, 1)
    queries = uniform_matrix(100, dim, 2)
    ref = orc.RefBruteForce(dim, metric)
    ref.add(base)
    bf = gpu.BruteForceIndex(dim, metric)
    bf.add(base)
    for k in (1, 10, 100):
        a = bf.search_batch(queries, k)
        b = ref.search_batch(queries, k)
        np.testing.assert_array_equal(a[2], b[2])
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_errors(gpu):
    bf = gpu.BruteForceIndex(2)
    bf.add(np.array([[1.0, 2.0]], np.float32))
    with pytest.raises(ValueError, match="query has dimension 1, index has 2"):
        bf.search([1.0], 1)
    with pytest.raises(ValueError, match="k must be positive"):
        bf.search([1.0, 2.0], 0)
    with pytest.raises(ValueError, match="must not contain NaN or inf"):
        bf.search_batch(np.array([[np.nan, 0.0]], np.float32), 1)
    with pytest.raises(ValueError, match="NaN or inf"):
        bf.add(np.array([[np.nan, 0.0]], np.float32))
    assert len(bf) == 1


@pytest.mark.parametrize("metric,make", [
    (0, "sift"), (2, "glove"), (1, "scaled"), (0, "uniform")])
def test_tensor_core_equals_exact_at_scale(gpu, metric, make):
    """Many tiles and chunks: the tensor-core path (with certification and the exact fallback)
    returns exactly the exact kernel's (= the reference's) ids and distance bits."""
    from hnsw_vector_search_b200 import datasets as ds
    if make == "sift":
        base, queries = ds.config_sift_like(rows=40_000, n_queries=600)
    elif make == "glove":
        base, queries = ds.config_glove_like(rows=30_000, n_queries=400)
    elif make == "scaled":
        base, queries = ds.config_scaled_ip(rows=30_000, n_queries=400)
    else:
        base, queries = uniform_matrix(25_000, 100, 7), uniform_matrix(300, 100, 8)
    bf = gpu.BruteForceIndex(base.shape[1], metric)
    bf.add(base)
    for k in (1, 10):
        a = bf.search_batch(queries, k, method="exact")
        b = bf.search_batch(queries, k, method="tensor_core")
        if make == "sift":
            assert gpu.BruteForceIndex.last_uncertified() == 0
        np.testing.assert_array_equal(a[2], b[2])
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("dim,nq", [(200, 1), (256, 129), (40, 3)])
@pytest.mark.parametrize("k", [1, 24, 48])
def test_tensor_core_equals_exact_across_shapes(gpu, dim, nq, k):
    """The shapes the work split and the MMA sequence specialize on: 1 to 4 K chunks of 64 (d 40,
    200, 256), a single query tile split into many short chunks (nq 1 or 3: each chunk a tile or
    two), candidate lists of 16, 32 and 64 (k 1, 24, 48) with their quarter-rank floors, integer
    data (exact scores) and real-valued data (lo terms, certification margins)."""
    for base, queries in ((integer_matrix(9_000, dim, 21), integer_matrix(nq, dim, 22)),
                          (uniform_matrix(9_000, dim, 23), uniform_matrix(nq, dim, 24))):
        bf = gpu.BruteForceIndex(dim)
        bf.add(base)
        a = bf.search_batch(queries, k, method="exact")
        b = bf.search_batch(queries, k, method="tensor_core")
        np.testing.assert_array_equal(a[2], b[2])
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_tensor_core_matches_reference(gpu, orc):
    from hnsw_vector_search_b200 import datasets as ds
    base, queries = ds.config_sift_like(rows=20_000, n_queries=200)
    ref = orc.RefBruteForce(128, 0)
    ref.add(base)
    bf = gpu.BruteForceIndex(128)
    bf.add(base)
    a = bf.search_batch(queries, 10, method="tensor_core")
    # Integer data: the tensor cores' scores are exact, so every query is certified and none
    # falls back to the exact kernel.
    assert gpu.BruteForceIndex.last_uncertified() == 0
    b = ref.search_batch(queries, 10)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("method", METHODS)
def test_concurrent_searches_with_different_k(gpu, method):
    """BruteForceIndex::search is const and safe from several threads; threads with k 1, 10 and
    40 launch with different shared-memory sizes on one device, and every result equals the same
    search run alone."""
    from concurrent.futures import ThreadPoolExecutor
    if not method_available(gpu, method):
        pytest.skip(f"{method} brute force is not available on this device")
    base = integer_matrix(20_000, 64, 5)
    queries = integer_matrix(256, 64, 6)
    bf = gpu.BruteForceIndex(64)
    bf.add(base)
    ks = [1, 10, 40]
    want = {k: bf.search_batch(queries, k, method=method) for k in ks}
    with ThreadPoolExecutor(max_workers=3) as pool:
        jobs = [(k, pool.submit(bf.search_batch, queries, k, method)) for _ in range(5) for k in ks]
        for k, job in jobs:
            got = job.result()
            np.testing.assert_array_equal(got[0], want[k][0])
            np.testing.assert_array_equal(got[1].view(np.uint32), want[k][1].view(np.uint32))


def test_tensor_core_timeout_releases_everything_and_the_next_call_succeeds(gpu):
    """The timeout path of the tensor-core kernel's bounded waits, made to run out on purpose
    without any fault: with a pipeline-wait limit of 1 ns every CTA gives up at its first wait
    for a copy or an MMA, drains its own copies and MMAs (those waits keep the full 1 s bound),
    frees its tensor memory and returns; the call reports VDX_ERR_DEVICE_TIMEOUT. With the
    default limit back, the next calls succeed with the exact results (tensor memory that was
    not freed would make later allocations fail or block)."""
    from hnsw_vector_search_b200 import datasets as ds
    base, queries = ds.config_sift_like(rows=20_000, n_queries=300)
    bf = gpu.BruteForceIndex(128)
    bf.add(base)
    want = bf.search_batch(queries, 10, method="exact")
    lib = gpu.lib()
    try:
        lib.vdx_testing_set_tc_wait_ns(1)
        with pytest.raises(gpu.DeviceTimeout, match="timed out"):
            bf.search_batch(queries, 10, method="tensor_core")
    finally:
        lib.vdx_testing_set_tc_wait_ns(0)
    for _ in range(3):
        got = bf.search_batch(queries, 10, method="tensor_core")
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1].view(np.uint32), want[1].view(np.uint32))
