"""The GPU-backed Python index (hnsw_vector_search_b200.knn.Index), against the reference's Python
binding contract (python/bindings.cpp:322-416, python/tests/test_index.py of the reference):
the input rules and errors run on the host; knn_query results equal the reference library's
search on the same graph (built the same way, so byte-identical)."""

import numpy as np
import pytest

DIM = 16


def vectors(n, dim=DIM, seed=0):
    return np.random.default_rng(seed).standard_normal((n, dim)).astype(np.float32)


@pytest.fixture
def Index(vdx):
    from hnsw_vector_search_b200.knn import Index
    return Index


# --- host side: construction, input rules, ids ------------------------------------------------

def test_add_items_returns_consecutive_int64_ids_and_properties(Index):
    index = Index("ip", 8, M=12, ef_construction=50)
    first = index.add_items(vectors(3, dim=8))
    second = index.add_items(vectors(2, dim=8, seed=1)[0])  # one 1-D vector
    assert first.dtype == np.int64 and list(first) == [0, 1, 2] and list(second) == [3]
    assert (index.space, index.dim, index.M, index.ef_construction, len(index)) == ("ip", 8, 12, 50, 4)
    assert index.memory_bytes() >= 4 * 8 * 4
    assert repr(index) == "<hnsw_vector_search_b200.Index space='ip' dim=8 M=12 ef_construction=50 ef=64 len=4>"


@pytest.mark.parametrize("dtype", [np.float64, np.float16, np.int32, ">f4"])
def test_other_dtypes_are_rejected_with_type_error(Index, dtype):
    index = Index("l2", DIM)
    with pytest.raises(TypeError, match=r"must be float32.*astype"):
        index.add_items(vectors(4).astype(dtype))
    with pytest.raises(TypeError, match="must be float32"):
        index.knn_query(vectors(4).astype(dtype))
    assert len(index) == 0


def test_non_buffers_non_contiguous_and_misshapen_inputs_are_rejected(Index):
    index = Index("l2", DIM)
    with pytest.raises(TypeError):
        index.add_items([[1.0] * DIM])
    for bad in (np.asfortranarray(vectors(8)), vectors(8)[::2], np.repeat(vectors(8), 2, axis=1)[:, ::2]):
        with pytest.raises(ValueError, match="C-contiguous"):
            index.add_items(bad)
        with pytest.raises(ValueError, match="C-contiguous"):
            index.knn_query(bad)
    raw = np.zeros(4 * DIM * 4 + 1, np.uint8)[1:].view(np.float32).reshape(4, DIM)
    with pytest.raises(ValueError, match="aligned"):
        index.add_items(raw)
    with pytest.raises(ValueError, match="1-D .* or 2-D"):
        index.add_items(np.zeros((2, 2, DIM), np.float32))
    with pytest.raises(ValueError, match="dimension"):
        index.add_items(vectors(2, dim=DIM + 1))
    assert len(index) == 0


def test_bad_values_and_arguments_raise_the_reference_errors(Index):
    index = Index("cosine", DIM)
    bad = vectors(3)
    bad[1, 2] = np.nan
    with pytest.raises(ValueError, match="NaN or inf"):
        index.add_items(bad)
    with pytest.raises(ValueError, match="zero"):
        index.add_items(np.zeros((1, DIM), np.float32))
    assert len(index) == 0
    for kwargs, message in (({"space": "euclidean"}, "space must be"), ({"dim": 0}, "dim must be positive"),
                            ({"M": 1}, "M must be at least 2"),
                            ({"ef_construction": 0}, "ef_construction must be positive")):
        with pytest.raises(ValueError, match=message):
            Index(**({"space": "l2", "dim": DIM} | kwargs))
    with pytest.raises(TypeError):
        Index("l2", DIM, seed=-1)
    index.add_items(vectors(10))
    for kwargs in ({"k": 0}, {"k": -1}, {"ef": 0}):
        with pytest.raises(ValueError, match="must be positive"):
            index.knn_query(vectors(2, seed=1), **kwargs)
    with pytest.raises(ValueError, match="ef must be positive"):
        index.set_ef(0)
    with pytest.raises(ValueError, match="ef must be positive"):
        index.ef = -5
    assert index.ef == 64
    with pytest.raises(ValueError, match="num_threads"):
        index.add_items(vectors(2), num_threads=-1)


def test_save_and_load_keep_the_graph(Index, tmp_path):
    index = Index("l2", DIM, M=8, ef_construction=40, seed=3)
    index.add_items(vectors(200))
    index.save(tmp_path / "a.vdx")
    again = Index.load(tmp_path / "a.vdx")
    assert (again.space, again.dim, again.M, again.ef_construction, len(again), again.ef) == ("l2", DIM, 8, 40, 200, 64)
    again.save(tmp_path / "b.vdx")
    assert (tmp_path / "a.vdx").read_bytes() == (tmp_path / "b.vdx").read_bytes()


# --- GPU: results ----------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("space", ["l2", "ip", "cosine"])
def test_knn_query_equals_the_reference_search(gpu, orc, Index, space, tmp_path):
    base, queries = vectors(2000, seed=4), vectors(100, seed=5)
    index = Index(space, DIM, M=8, ef_construction=64, seed=9)
    index.add_items(base)                          # one thread: the reference's serial graph
    ref = orc.RefHnsw(DIM, {"l2": 0, "ip": 1, "cosine": 2}[space], 8, 64, 9)
    ref.add(base, threads=1)
    for k, ef in ((1, 1), (10, 32), (10, None), (7, 300)):
        ids, d = index.knn_query(queries, k=k, ef=ef)
        assert ids.dtype == np.int64 and d.dtype == np.float32 and ids.shape == (100, k)
        want_ids, want_d, _ = ref.search_batch(queries, k, 64 if ef is None else ef, 1)
        np.testing.assert_array_equal(ids, want_ids.astype(np.int64))
        np.testing.assert_array_equal(d.view(np.uint32), want_d.view(np.uint32))


@pytest.mark.gpu
def test_padding_empty_index_and_default_ef(gpu, Index):
    small = Index("l2", DIM)
    small.add_items(vectors(5))
    ids, d = small.knn_query(vectors(5)[:2], k=8)
    assert sorted(ids[0, :5]) == [0, 1, 2, 3, 4]
    np.testing.assert_array_equal(ids[:, 5:], -1)
    np.testing.assert_array_equal(d[:, 5:], np.inf)
    empty = Index("cosine", DIM)
    ids, d = empty.knn_query(vectors(3), k=4)
    np.testing.assert_array_equal(ids, np.full((3, 4), -1))
    np.testing.assert_array_equal(d, np.full((3, 4), np.inf, np.float32))
    ids, d = empty.knn_query(np.empty((0, DIM), np.float32), k=4)
    assert ids.shape == d.shape == (0, 4)
    sparse = Index("l2", DIM, M=4, ef_construction=8)
    sparse.add_items(vectors(1000))
    q = vectors(50, seed=1)
    sparse.ef = 10
    narrow, _ = sparse.knn_query(q, k=10)
    np.testing.assert_array_equal(narrow, sparse.knn_query(q, k=10, ef=10)[0])
    wide, _ = sparse.knn_query(q, k=10, ef=400)
    assert not np.array_equal(narrow, wide)
    empty.add_items(vectors(3))
    with pytest.raises(ValueError, match="zero"):
        empty.knn_query(np.zeros(DIM, np.float32))
