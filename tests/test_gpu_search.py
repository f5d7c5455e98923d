"""GPU HNSW search through the C ABI against the reference: published fingerprints, golden
results, bit-exact ids and distances on reference-built graphs for every metric, the reference's
error behaviour, and the device counters against the oracle's."""

from pathlib import Path

import numpy as np
import pytest

from conftest import integer_matrix, uniform_matrix

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FINGERPRINT_GREEDY = 6133164406513967666
FINGERPRINT_TOP10 = 15666754926265556722


def assert_same(a, b, what=""):
    np.testing.assert_array_equal(a[2], b[2], err_msg=f"counts {what}")
    np.testing.assert_array_equal(a[0], b[0], err_msg=f"ids {what}")
    np.testing.assert_array_equal(np.asarray(a[1]).view(np.uint32), np.asarray(b[1]).view(np.uint32),
                                  err_msg=f"distances {what}")


def test_gpu_reproduces_published_fingerprints(gpu, orc):
    ix = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    queries = integer_matrix(200, 16, 2)
    o = orc.Oracle()
    assert o.fingerprint(*ix.search_batch(queries, 1, 1)) == FINGERPRINT_GREEDY
    assert o.fingerprint(*ix.search_batch(queries, 10, 10)) == FINGERPRINT_TOP10


@pytest.mark.parametrize("k,ef", [(1, 1), (10, 10), (10, 40), (10, 200)])
def test_gpu_matches_golden_results(gpu, k, ef):
    g = np.load(GOLDEN / "kat_results.npz")
    ix = gpu.HnswIndex.load(GOLDEN / "kat_m8.vdx")
    got = ix.search_batch(integer_matrix(200, 16, 2), k, ef)
    assert_same(got, (g[f"ids_{k}_{ef}"], g[f"dists_{k}_{ef}"], g[f"counts_{k}_{ef}"]), f"k{k} ef{ef}")


@pytest.fixture(scope="module")
def small_l2(orc, tmp_path_factory):
    """The CPU-runnable workload: 10,000 x 128 integer L2, M 16, ef_construction 200, serial
    reference build, saved and loaded."""
    from hnsw_vector_search_b200.datasets import config_small_l2
    base, queries = config_small_l2()
    path = tmp_path_factory.mktemp("small") / "small.vdx"
    ref = orc.RefHnsw(128, 0, 16, 200, 42)
    ref.add(base, threads=0)
    ref.save(path)
    return path, base, queries


@pytest.mark.parametrize("ef", [16, 64, 128, 300, 700])
def test_gpu_equals_reference_on_small_l2(gpu, orc, small_l2, ef):
    """ef 300 and 700 (result capacity 512 and 1024) run with the global visited filter."""
    path, base, queries = small_l2
    ref = orc.RefHnsw.load(path)
    ix = gpu.HnswIndex.load(path)
    assert_same(ix.search_batch(queries, 10, ef), ref.search_batch(queries, 10, ef), f"ef {ef}")


def test_gpu_counters_equal_the_oracles(gpu, orc, small_l2):
    """Expansions and distance evaluations counted on the device equal the restatement's counts
    (no visited-filter misses at this size), so the roofline's byte counts are the algorithm's."""
    path, base, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    ix.search_batch(queries, 10, 64)
    st = gpu.HnswIndex.last_stats()
    _, _, _, ost = orc.OracleIndex(path).search_batch(queries, 10, 64, stats=True)
    assert st["queries"] == len(queries)
    assert st["expansions"] == int(ost[:, 0].sum())
    assert st["dist_layer0"] == int(ost[:, 1].sum())
    assert st["dist_upper"] == int(ost[:, 2].sum())
    assert st["duplicates"] == 0


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [16, 13, 100, 40, 128])
def test_gpu_equals_reference_on_real_valued_data(gpu, orc, tmp_path, metric, dim):
    base = uniform_matrix(1500, dim, 1)
    queries = uniform_matrix(80, dim, 2)
    ref = orc.RefHnsw(dim, metric, 8, 40, 42)
    ref.add(base, threads=0)
    ref.save(tmp_path / "g.vdx")
    ref = orc.RefHnsw.load(tmp_path / "g.vdx")
    ix = gpu.HnswIndex.load(tmp_path / "g.vdx")
    for k, ef in [(1, 1), (10, 10), (10, 40), (10, 200)]:
        assert_same(ix.search_batch(queries, k, ef), ref.search_batch(queries, k, ef),
                    f"metric {metric} dim {dim} k {k} ef {ef}")


def test_batch_equals_single_searches(gpu, tmp_path):
    base = integer_matrix(1000, 16, 1)
    queries = integer_matrix(100, 16, 3)
    for metric in ("l2", "cosine"):
        ix = gpu.HnswIndex(16, metric, M=8, ef_construction=64)
        ix.add(base)
        ids, d, c = ix.search_batch(queries, 10, 32)
        for q in range(len(queries)):
            one = ix.search(queries[q], 10, 32)
            assert one == [(float(d[q, i]), int(ids[q, i])) for i in range(c[q])]


def test_concurrent_searches_with_different_layouts(gpu, small_l2):
    """search_batch is safe from several threads at once (include/vecdex/hnsw.hpp:58-62 of the
    reference). Threads searching at ef 16 / 64 / 128 / 300 launch the kernel with different
    shared-memory layouts on one device; every result equals the same search run alone."""
    from concurrent.futures import ThreadPoolExecutor
    path, _, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    q = queries[:300]
    efs = [16, 64, 128, 300]
    want = {ef: ix.search_batch(q, 10, ef) for ef in efs}
    with ThreadPoolExecutor(max_workers=4) as pool:
        jobs = [(ef, pool.submit(ix.search_batch, q, 10, ef)) for _ in range(6) for ef in efs]
        for ef, job in jobs:
            assert_same(job.result(), want[ef], f"ef {ef}")


def test_exact_when_ef_covers_every_node(gpu, orc):
    base = uniform_matrix(300, 8, 1)
    queries = uniform_matrix(20, 8, 2)
    ix = gpu.HnswIndex(8, "l2", M=8, ef_construction=50)
    ix.add(base)
    assert ix.inspect()["reachable"] == 300
    got = ix.search_batch(queries, 10, 300)
    want = orc.Oracle().bruteforce(base, queries, 10)
    assert_same(got, want, "ef = n")
    got = ix.search_batch(queries, 10, 100000)  # ef far above n: the same exhaustive search
    assert_same(got, want, "ef >> n")


def test_returns_everything_when_k_exceeds_size(gpu, orc):
    base = uniform_matrix(5, 4, 1)
    ix = gpu.HnswIndex(4, "l2", M=4, ef_construction=10)
    ix.add(base)
    q = np.array([[0.1, 0.2, 0.3, 0.4]], np.float32)
    ids, d, c = ix.search_batch(q, 10, 10)
    want = orc.Oracle().bruteforce(base, q, 10)
    assert c[0] == 5
    assert_same((ids, d, c), want)
    assert list(ids[0, 5:]) == [0xFFFFFFFF] * 5 and np.all(np.isinf(d[0, 5:]))


def test_empty_index_and_empty_batch(gpu):
    empty = gpu.HnswIndex(4)
    ids, d, c = empty.search_batch(integer_matrix(5, 4, 1), 3, 10)
    assert list(c) == [0] * 5
    assert empty.search([1.0, 2.0, 3.0, 4.0], 5, 10) == []
    ix = gpu.HnswIndex(4, M=4, ef_construction=16)
    ix.add(integer_matrix(50, 4, 2))
    ids, d, c = ix.search_batch(np.zeros((0, 4), np.float32), 3, 10)
    assert ids.shape == (0, 3)


def test_single_node(gpu):
    ix = gpu.HnswIndex(3)
    ix.add_one([1.0, 2.0, 3.0])
    assert ix.search([1.0, 2.0, 3.0], 1, 1) == [(0.0, 0)]


def test_duplicates(gpu):
    same = [0.5, -0.5, 0.25, 1.0]
    ix = gpu.HnswIndex(4, "l2", M=8, ef_construction=40)
    for _ in range(100):
        ix.add_one(same)
    ix.add(uniform_matrix(100, 4, 6))
    found = ix.search(same, 10, 50)
    assert len(found) == 10
    assert all(d == 0.0 and i < 100 for d, i in found)


def test_bad_queries_raise_the_reference_errors(gpu):
    ix = gpu.HnswIndex(4, "l2", M=8, ef_construction=32)
    ix.add(integer_matrix(200, 4, 1))
    q = integer_matrix(64, 4, 2)
    with pytest.raises(ValueError, match="HnswIndex::search_batch: k must be positive"):
        ix.search_batch(q, 0, 10)
    with pytest.raises(ValueError, match="query has dimension 3, index has 4"):
        ix.search_batch(integer_matrix(8, 3, 2), 5, 10)
    q[37, 2] = np.nan
    with pytest.raises(ValueError, match="HnswIndex::search_batch: query must not contain NaN or inf"):
        ix.search_batch(q, 5, 10)
    q[37, 2] = np.inf
    with pytest.raises(ValueError, match="must not contain NaN or inf"):
        ix.search_batch(q, 5, 10)
    cos = gpu.HnswIndex(2, "cosine", M=4, ef_construction=8)
    cos.add(uniform_matrix(20, 2, 1))
    with pytest.raises(ValueError, match="can't normalize a zero query"):
        cos.search_batch(np.zeros((3, 2), np.float32), 2, 5)
    with pytest.raises(ValueError, match="HnswIndex::search: can't normalize|the cosine metric"):
        cos.search([0.0, 0.0], 2, 5)
    # The index is still usable after a rejected call.
    ids, d, c = ix.search_batch(integer_matrix(4, 4, 9), 5, 10)
    assert list(c) == [5] * 4


def test_page_locked_queries_are_read_in_place_with_the_same_results(gpu, orc, small_l2):
    """Queries in page-locked host memory are read by the kernel across the bus instead of being
    copied first: same bits as pageable queries and as the reference, same error reports."""
    import torch
    path, _, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    ref = orc.RefHnsw.load(path)
    pinned = torch.from_numpy(queries).pin_memory()
    for precision in ("fp32", "bf16"):
        o = {} if precision == "fp32" else {"precision": "bf16", "rerank": 40}
        assert_same(ix.search_batch(pinned.numpy(), 10, 36, **o), ix.search_batch(queries.copy(), 10, 36, **o),
                    precision)
    assert_same(ix.search_batch(pinned.numpy()[17:530], 10, 64), ref.search_batch(queries[17:530], 10, 64, 1),
                "pinned slice vs reference")
    # Results written in place into page-locked buffers, and into pageable ones passed as out=.
    nq = len(queries)
    for make in (lambda t: t.pin_memory().numpy(), lambda t: t.numpy()):
        out = (make(torch.full((nq, 10), 7, dtype=torch.int32)).view(np.uint32),
               make(torch.full((nq, 10), 7.0)), make(torch.full((nq,), 7, dtype=torch.int32)).view(np.uint32))
        got = ix.search_batch(pinned.numpy(), 10, 36, out=out)
        assert all(g is o for g, o in zip(got, out))
        assert_same(out, ref.search_batch(queries, 10, 36, 1), "out=")
    with pytest.raises(ValueError, match="out distances must be"):
        ix.search_batch(queries, 10, 36, out=(out[0], np.empty((nq, 10), np.float64), out[2]))
    with pytest.raises(ValueError, match="out ids must be"):
        ix.search_batch(queries, 10, 36, out=(out[0][:, :5], out[1], out[2]))
    pinned[37, 2] = float("nan")
    with pytest.raises(ValueError, match="query must not contain NaN or inf"):
        ix.search_batch(pinned.numpy(), 10, 36)
    cos = gpu.HnswIndex(2, "cosine", M=4, ef_construction=8)
    cos.add(uniform_matrix(20, 2, 1))
    with pytest.raises(ValueError, match="can't normalize a zero query"):
        cos.search_batch(torch.zeros((3, 2)).pin_memory().numpy(), 2, 5)


def test_bf16_traversal_is_exact_on_integer_data(gpu, small_l2):
    """Integers up to 256 are exact in bfloat16, so the BF16 traversal scores exactly what FP32
    scores and the results are the FP32 (reference) results."""
    path, base, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    for ef in (16, 64):
        assert_same(ix.search_batch(queries, 10, ef, precision="bf16"),
                    ix.search_batch(queries, 10, ef), f"bf16 ef {ef}")


def test_fp8_traversal_with_rerank_keeps_recall(gpu, orc, small_l2):
    path, base, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    truth, _, _ = orc.Oracle().bruteforce(base, queries, 10)
    ids32, _, _ = ix.search_batch(queries, 10, 64)
    ids8, d8, _ = ix.search_batch(queries, 10, 64, precision="fp8", rerank=40)

    def recall(ids):
        return np.mean([len(set(a) & set(b)) / 10 for a, b in zip(ids, truth)])

    assert recall(ids8) >= recall(ids32) - 0.02
    # Re-ranked distances are exact FP32 distances of the returned ids.
    o = orc.Oracle()
    for q in range(0, len(queries), 97):
        for i in range(10):
            assert np.float32(o.l2(queries[q], base[ids8[q, i]])) == d8[q, i]


def _stored_rows(orc, base, metric):
    """The rows as the index stores them: normalized in the reference's order under cosine."""
    rows = np.array(base, np.float32, copy=True)
    if metric == 2:
        for r in rows:
            orc.Oracle().L.vo_normalize(r.ctypes.data, r.size)
    return rows


def _exact(orc, metric, q, row):
    o = orc.Oracle()
    return np.float32(o.l2(q, row)) if metric == 0 else np.float32(1.0) - np.float32(o.ip(q, row))


@pytest.mark.parametrize("precision", ["bf16", "fp8"])
@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [40, 128])
def test_low_precision_traversal_equals_the_quantized_oracle(gpu, orc, tmp_path, precision, metric, dim):
    """BF16 / FP8 traversal on real-valued data, bit for bit. The oracle quantizes the stored
    rows as the GPU does (round to nearest even; E4M3 with the per-row FP32 scale max|x| / 448)
    and runs the reference's search on them: with rerank="none" the GPU returns exactly those ids
    and distances. With a re-rank of r, the GPU's result is the oracle's best min(r, ef)
    candidates re-scored with the exact FP32 distance in the reference's order, best k by
    (distance, id). Dimension 128 runs the kernels' unrolled distance routines (two lanes a row,
    and four lanes a row in rounds of at most 8 rows); real-valued data checks their order."""
    base = uniform_matrix(2000, dim, 11)
    queries = uniform_matrix(120, dim, 12)
    ref = orc.RefHnsw(dim, metric, 8, 60, 42)
    ref.add(base, threads=0)
    ref.save(tmp_path / "g.vdx")
    ix = gpu.HnswIndex.load(tmp_path / "g.vdx")
    quant = orc.OracleIndex(tmp_path / "g.vdx")
    quant.quantize(precision)
    stored = _stored_rows(orc, base, metric)
    for k, ef in [(1, 1), (10, 10), (10, 40), (10, 150)]:
        got = ix.search_batch(queries, k, ef, precision=precision, rerank="none")
        want = quant.search_batch(queries, k, ef)
        assert_same(got, want[:3], f"{precision} metric {metric} k {k} ef {ef}")
    k, ef, r = 10, 64, 24
    ids, d, c = ix.search_batch(queries, k, ef, precision=precision, rerank=r)
    cand, _, cc = quant.search_batch(queries, min(r, ef), ef)[:3]
    for qi in range(len(queries)):
        q = np.array(queries[qi], np.float32, copy=True)
        if metric == 2:
            orc.Oracle().L.vo_normalize(q.ctypes.data, q.size)
        scored = sorted((_exact(orc, metric, q, stored[i]), int(i)) for i in cand[qi, :cc[qi]])[:k]
        assert c[qi] == len(scored)
        assert [i for _, i in scored] == ids[qi, :c[qi]].tolist(), f"query {qi}"
        assert np.array([x for x, _ in scored], np.float32).view(np.uint32).tolist() == \
            d[qi, :c[qi]].view(np.uint32).tolist(), f"query {qi}"


def test_device_api_with_per_query_k_and_ef(gpu, small_l2):
    torch = pytest.importorskip("torch")
    path, base, queries = small_l2
    ix = gpu.HnswIndex.load(path)
    nq = 256
    rng = np.random.default_rng(5)
    ks = rng.choice([1, 10, 32], size=nq).astype(np.uint32)
    efs = (ks + rng.integers(0, 100, size=nq)).astype(np.uint32)
    dev = torch.device("cuda:0")
    q = torch.from_numpy(queries[:nq]).to(dev)
    k_t = torch.from_numpy(ks.astype(np.int32)).to(dev)
    ef_t = torch.from_numpy(efs.astype(np.int32)).to(dev)
    width = 32
    ids = torch.empty((nq, width), dtype=torch.int32, device=dev)
    d = torch.empty((nq, width), dtype=torch.float32, device=dev)
    c = torch.empty(nq, dtype=torch.int32, device=dev)
    work = torch.zeros(int(gpu.lib().vdx_work_words()), dtype=torch.int32, device=dev)
    ix.search_batch_device(q, 32, int(efs.max()), width, ids, d, c, work,
                           k_per_query=k_t, ef_per_query=ef_t,
                           stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(work[0].item()) == 0
    ids, d, c = ids.cpu().numpy().view(np.uint32), d.cpu().numpy(), c.cpu().numpy().view(np.uint32)
    for qi in range(0, nq, 17):
        want = ix.search_batch(queries[qi:qi + 1], int(ks[qi]), int(efs[qi]))
        assert c[qi] == want[2][0]
        np.testing.assert_array_equal(ids[qi, :ks[qi]], want[0][0])
        np.testing.assert_array_equal(d[qi, :ks[qi]], want[1][0])
