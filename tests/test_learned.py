"""Learned early termination: the FP64 CPU oracle of the network pinned by finite differences,
the GPU forward / backward / Adam kernels checked against it, the training traces, and what the
trained network gains over the plain search at equal recall."""

import json
from pathlib import Path

import numpy as np
import pytest

import mlp_oracle as mo
from conftest import integer_matrix

GOLDEN = Path(__file__).resolve().parent / "golden"


def random_net(seed=0):
    g = np.random.default_rng(seed)
    w = (g.standard_normal(mo.N_PARAMS) * 0.2).astype(np.float32)
    x = g.standard_normal((300, mo.F)).astype(np.float32)
    y = (g.random(300) < 0.4).astype(np.float32)
    return w, x, y


def test_oracle_gradient_matches_finite_differences():
    w, x, y = random_net(1)
    loss, g = mo.loss_and_grad(x, y, w)
    wq = mo.rounded(w).astype(np.float64)
    rng = np.random.default_rng(2)
    for i in rng.choice(mo.N_PARAMS, size=60, replace=False):
        h = 1e-7  # small enough that no ReLU input crosses zero within the step
        wp, wm = wq.copy(), wq.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mo.loss_only(x, y, wp) - mo.loss_only(x, y, wm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    torch = pytest.importorskip("torch")
    v = np.random.default_rng(3).standard_normal(100000).astype(np.float32) * 10
    want = torch.from_numpy(v).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(mo.bf16_round(v), want)


@pytest.mark.gpu
def test_gpu_gradients_match_the_fp64_oracle(gpu):
    from hnsw_vector_search_b200 import learned
    w, x, y = random_net(4)
    loss, g = learned.gradient(x, y, w)
    ref_loss, ref = mo.loss_and_grad(x, y, w)
    assert abs(loss - ref_loss) <= 1e-5 * (1 + abs(ref_loss))
    err = np.abs(g - ref)
    scale = np.abs(ref).max()
    assert err.max() <= 1e-4 * scale, (err.max(), scale)
    # Every block of parameters is checked, not only the largest entries.
    for lo, hi in ((mo.OFF_W1, mo.OFF_B1), (mo.OFF_B1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_B2),
                   (mo.OFF_B2, mo.OFF_W3), (mo.OFF_W3, mo.OFF_B3)):
        np.testing.assert_allclose(g[lo:hi], ref[lo:hi], rtol=1e-3, atol=1e-4 * scale)


@pytest.mark.gpu
def test_gpu_training_learns_and_probabilities_match_the_oracle(gpu):
    from hnsw_vector_search_b200 import learned
    g = np.random.default_rng(5)
    x = g.standard_normal((20000, mo.F)).astype(np.float32) * 3 + 1
    y = (x[:, 0] + 0.5 * x[:, 3] - x[:, 7] > 1.0).astype(np.float32)
    model, losses = learned.train(x, y, np.zeros((4, 8), np.float32), epochs=6, batch=1024)
    assert losses[-1] < 0.5 * losses[0], losses
    p = learned.probabilities(model, x[:500])
    want = mo.probabilities(x[:500], model.weights, model.mean, model.inv_std)
    np.testing.assert_allclose(p, want, atol=1e-4)
    acc = np.mean((p > 0.5) == (y[:500] > 0.5))
    assert acc > 0.95


@pytest.fixture(scope="module")
def small_graph(tmp_path_factory):
    import hnsw_vector_search_b200 as v
    from hnsw_vector_search_b200.datasets import integer_clusters
    base = integer_clusters(10_000, 128, 100, seed=1, centers_seed=101, sigma=12.0)
    ix = v.HnswIndex(128, "l2", M=16, ef_construction=200)
    ix.add(base, num_threads=0)
    return ix, base


def truth_of(v, base, queries, k=10):
    bf = v.BruteForceIndex(base.shape[1])
    bf.add(base)
    ids, _, _ = bf.search_batch(queries, k)
    return ids


@pytest.mark.gpu
def test_traces_are_consistent_with_the_plain_search(gpu, small_graph):
    from hnsw_vector_search_b200 import learned
    from hnsw_vector_search_b200.datasets import integer_clusters
    ix, base = small_graph
    q = integer_clusters(500, 128, 100, seed=21, centers_seed=101, sigma=12.0)
    truth = truth_of(gpu, base, q)
    tr = learned.traces(ix, q, truth, k=10, ef=128)
    ids, _, _ = ix.search_batch(q, 10, 128)
    hits = [len(set(a.tolist()) & set(b.tolist())) for a, b in zip(ids, truth)]
    np.testing.assert_array_equal(tr["final"], hits)
    assert tr["points"].min() >= 16  # ef 128 expands at least 128 nodes: 16 checkpoints
    assert np.all(tr["hits"][:, 0] <= tr["final"] + 10)
    st = gpu.HnswIndex.last_stats()
    assert np.isfinite(tr["features"][tr["points"] > 0][:, :4]).all()


@pytest.fixture(scope="module")
def mixed_workload(gpu):
    """200,000 x 128 SIFT-like base (1,000 anisotropic clusters); queries from the same mixture,
    half of them pushed between the clusters (noise sigma 45), so query difficulty varies."""
    from hnsw_vector_search_b200.datasets import integer_clusters, mixed_difficulty
    base = integer_clusters(200_000, 128, 1000, seed=1, centers_seed=111)
    ix = gpu.HnswIndex(128, "l2", M=16, ef_construction=200)
    ix.add(base, num_threads=0)
    bf = gpu.BruteForceIndex(128)
    bf.add(base)

    def queries(n, seed):
        q = integer_clusters(n, 128, 1000, seed=seed, centers_seed=111)
        return mixed_difficulty(q, 0.5, 45.0, seed=seed + 1000)
    return ix, bf, queries


@pytest.mark.gpu
def test_learned_stop_gains_over_plain_search_at_equal_recall(gpu, mixed_workload):
    """Trained on traces at its ef cap (192) for 20,000 queries, its threshold calibrated on
    3,000 others for recall@10 0.96, evaluated on a third set of 5,000: the learned stop reaches
    the recall with fewer layer-0 distance evaluations than the plain search needs for the same
    recall (interpolated along the plain search's ef sweep)."""
    from hnsw_vector_search_b200 import learned
    ix, bf, queries = mixed_workload
    train_q, cal_q, test_q = queries(20_000, 21), queries(3_000, 22), queries(5_000, 23)
    truth = lambda q: bf.search_batch(q, 10, method="tensor_core")[0]  # noqa: E731
    cap, target = 192, 0.96
    tr = learned.traces(ix, train_q, truth(train_q), k=10, ef=cap)
    x, y = learned.training_set(tr)
    model, losses = learned.train(x, y, tr["proj"], epochs=6)
    assert losses[-1] < losses[0]

    test_truth = truth(test_q)
    plain = []
    for ef in (24, 32, 40, 48, 64, 96, 128, 192, 256):
        ids, _, _ = ix.search_batch(test_q, 10, ef)
        plain.append((learned.recall(ids, test_truth, 10), gpu.HnswIndex.last_stats()["dist_layer0"]))
    thr, _ = learned.calibrate(ix, model, cal_q, truth(cal_q), 10, target, cap)
    ids, _, _ = ix.search_batch(test_q, 10, cap, learned_stop=True, stop_threshold=thr)
    rec = learned.recall(ids, test_truth, 10)
    work = gpu.HnswIndex.last_stats()["dist_layer0"]
    plain.sort()
    plain_work = None
    for (r0, w0), (r1, w1) in zip(plain, plain[1:]):
        if r0 <= rec <= r1:
            plain_work = w0 + (w1 - w0) * (rec - r0) / max(r1 - r0, 1e-12)
    report = {"recall_learned": rec, "work_learned": work, "threshold": thr, "plain": plain,
              "plain_work_at_equal_recall": plain_work,
              "gain": None if plain_work is None else plain_work / work}
    print(json.dumps(report))
    assert rec >= target - 0.01, report
    assert plain_work is not None and plain_work / work >= 1.08, report
