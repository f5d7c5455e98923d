"""The batched GPU graph build (HnswIndex::add_gpu) against the reference's acceptance bar for a
parallel build (tests/hnsw_parallel_test.cpp:106-136 of the reference): a healthy graph (no
broken invariant, at most 1 node in 1000 unreachable), the serial build's top layer (levels are
drawn in the serial order), and recall@10 at most 0.005 below the serial build's."""

import numpy as np
import pytest

from conftest import integer_matrix

pytestmark = pytest.mark.gpu


def recall(ids, truth, k=10):
    return float(np.mean([len(set(a[:k].tolist()) & set(b[:k].tolist())) / k for a, b in zip(ids, truth)]))


def check_gpu_build(gpu, base, queries, M, efc, ef, metric="l2"):
    serial = gpu.HnswIndex(base.shape[1], metric, M=M, ef_construction=efc, seed=42)
    serial.add(base, num_threads=1)
    built = gpu.HnswIndex(base.shape[1], metric, M=M, ef_construction=efc, seed=42)
    built.add(base, device=0)
    report = built.inspect()
    serial_report = serial.inspect()
    assert report["first_violation"] == "" and report["violations"] == 0, report
    # At most 1 node in 1000 unreachable beyond what the serial build leaves (inner product is
    # not a metric, and even a serial build orphans a few nodes there).
    allowed = min(len(base), serial_report["reachable"]) - len(base) // 1000
    assert report["reachable"] >= allowed, (report, serial_report)
    assert report["max_level"] == serial_report["max_level"]
    bf = gpu.BruteForceIndex(base.shape[1], metric)
    bf.add(base)
    truth, _, _ = bf.search_batch(queries, 10)
    r_serial = recall(serial.search_batch(queries, 10, ef)[0], truth)
    r_gpu = recall(built.search_batch(queries, 10, ef)[0], truth)
    print(f"{metric}: serial {r_serial:.4f} gpu {r_gpu:.4f}, reachable {serial_report['reachable']} / "
          f"{report['reachable']} of {len(base)}")
    assert r_gpu >= r_serial - 0.005, (r_serial, r_gpu)
    return built


def test_gpu_build_matches_serial_recall_on_random_data(gpu):
    check_gpu_build(gpu, integer_matrix(2000, 16, 1), integer_matrix(1000, 16, 2), M=16, efc=64, ef=16)


def test_gpu_build_matches_serial_recall_on_clustered_data(gpu):
    from hnsw_vector_search_b200.datasets import integer_clusters
    base = integer_clusters(20_000, 128, 100, seed=1, centers_seed=101, sigma=12.0)
    queries = integer_clusters(1000, 128, 100, seed=2, centers_seed=101, sigma=12.0)
    check_gpu_build(gpu, base, queries, M=16, efc=200, ef=32)


@pytest.mark.parametrize("metric", ["ip", "cosine"])
def test_gpu_build_other_metrics(gpu, metric):
    g = np.random.default_rng(3)
    base = g.standard_normal((6000, 24)).astype(np.float32)
    queries = g.standard_normal((500, 24)).astype(np.float32)
    check_gpu_build(gpu, base, queries, M=12, efc=80, ef=32, metric=metric)


def test_gpu_build_extends_an_index_and_its_device_copy_is_the_saved_graph(gpu, tmp_path):
    base = integer_matrix(5000, 16, 1)
    queries = integer_matrix(300, 16, 2)
    ix = gpu.HnswIndex(16, "l2", M=8, ef_construction=64)
    ix.add(base[:3000], num_threads=1)
    ix.add(base[3000:], device=0)
    assert len(ix) == 5000
    report = ix.inspect()
    assert report["violations"] == 0 and report["reachable"] >= 4995, report
    # The device mirror was built in place: its results equal those of the saved host graph.
    got = ix.search_batch(queries, 10, 40)
    ix.save(tmp_path / "g.vdx")
    again = gpu.HnswIndex.load(tmp_path / "g.vdx")
    want = again.search_batch(queries, 10, 40)
    for x, y in zip(got, want):
        np.testing.assert_array_equal(x, y)
