"""Recall measures used by the bench and the learned-stop training: the known answers of the
reference's tests/recall_test.cpp:28-100, restated as batches."""

import numpy as np
import pytest

from hnsw_vector_search_b200.recall import recall_at_k, threshold_recall_at_k


def one(found, truth, k):
    return recall_at_k([np.array(found, np.int64)], np.array([truth]), k)


def test_perfect_partial_and_zero():
    truth = [4, 8, 15, 16]
    assert one([4, 8, 15, 16], truth, 4) == 1.0
    assert one([16, 15, 8, 4], truth, 4) == 1.0  # order is ignored
    assert one([4, 99, 15, 98], truth, 4) == 0.5
    assert one([1, 2, 3, 5], truth, 4) == 0.0


def test_only_the_first_k_of_each_list_count():
    assert one([4, 15, 8], [4, 8, 15, 16], 2) == 0.5


def test_missing_and_duplicate_results():
    assert one([2, 1], [1, 2, 3, 4], 4) == 0.5
    assert one([], [1, 2, 3, 4], 4) == 0.0
    assert one([7, 7, 7], [7, 8, 9], 3) == pytest.approx(1.0 / 3.0)
    # the library's padding never matches a true id
    assert recall_at_k(np.array([[1, 0xFFFFFFFF]], np.uint32), np.array([[1, 2]]), 2) == 0.5


def test_bad_arguments():
    with pytest.raises(ValueError):
        one([1], [1, 2], 0)
    with pytest.raises(ValueError):
        one([1], [1, 2], 3)


def thr(dists, kth, k, tol=1e-5):
    return threshold_recall_at_k([np.array(dists, np.float32)], [kth], k, tol)


def test_threshold_recall_counts_ties_and_misses():
    assert thr([1, 2, 5], 5.0, 3) == 1.0
    assert thr([1, 2, 6], 5.0, 3) == pytest.approx(2.0 / 3.0)
    assert thr([7, 8, 9], 5.0, 3) == 0.0
    assert thr([1, 9, 2], 5.0, 2) == 0.5
    assert thr([1], 5.0, 4) == 0.25
    assert thr([], 5.0, 4) == 0.0


def test_threshold_tolerance_is_relative_above_one_and_absolute_below():
    assert thr([100000.5], 100000.0, 1) == 1.0
    assert thr([100002.0], 100000.0, 1) == 0.0
    assert thr([5e-6], 0.0, 1) == 1.0
    assert thr([5e-5], 0.0, 1) == 0.0
    assert thr([100000.5], 100000.0, 1, 0.0) == 0.0
    with pytest.raises(ValueError):
        thr([1], float("inf"), 1)
    with pytest.raises(ValueError):
        thr([1], 1.0, 1, -1.0)


def test_batch_equals_per_query_mean():
    rng = np.random.default_rng(3)
    truth = np.stack([rng.permutation(50)[:10] for _ in range(40)])
    found = np.stack([rng.permutation(50)[:10] for _ in range(40)]).astype(np.uint32)
    per = [len(set(found[i].tolist()) & set(truth[i].tolist())) / 10 for i in range(40)]
    assert recall_at_k(found, truth, 10) == pytest.approx(np.mean(per))
