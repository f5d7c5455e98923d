"""The oracle pinned: the reference library compiled here, and this repository's C restatement,
against the reference's own published known answers and against each other (CPU only)."""

from pathlib import Path

import numpy as np
import pytest

from conftest import integer_matrix, uniform_matrix

GOLDEN = Path(__file__).resolve().parent / "golden"

# tests/hnsw_parallel_test.cpp:164-167 of the reference.
FINGERPRINT_GREEDY = 6133164406513967666
FINGERPRINT_TOP10 = 15666754926265556722


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "kat_results.npz")


def test_reference_reproduces_its_published_fingerprints(orc):
    ref = orc.RefHnsw.load(GOLDEN / "kat_m8.vdx")
    queries = integer_matrix(200, 16, 2)
    o = orc.Oracle()
    ids, d, c = ref.search_batch(queries, 1, 1)
    assert o.fingerprint(ids, d, c) == FINGERPRINT_GREEDY
    ids, d, c = ref.search_batch(queries, 10, 10)
    assert o.fingerprint(ids, d, c) == FINGERPRINT_TOP10
    rep = ref.inspect()
    assert rep["max_level"] == 3
    assert round(rep["mean_degree0"] * 1000) == 11157


def test_reference_serial_build_is_the_published_graph(orc, tmp_path):
    """Building the fixture again, serially and one vector at a time, gives the same file."""
    base = integer_matrix(1000, 16, 1)
    a = orc.RefHnsw(16, 0, 8, 64, 42)
    a.add(base, threads=1)
    a.save(tmp_path / "a.vdx")
    b = orc.RefHnsw(16, 0, 8, 64, 42)
    for row in base:
        b.add_one(row)
    b.save(tmp_path / "b.vdx")
    golden = (GOLDEN / "kat_m8.vdx").read_bytes()
    assert (tmp_path / "a.vdx").read_bytes() == golden
    assert (tmp_path / "b.vdx").read_bytes() == golden


def test_oracle_reproduces_published_fingerprints(orc):
    ix = orc.OracleIndex(GOLDEN / "kat_m8.vdx")
    queries = integer_matrix(200, 16, 2)
    o = orc.Oracle()
    assert o.fingerprint(*ix.search_batch(queries, 1, 1)) == FINGERPRINT_GREEDY
    assert o.fingerprint(*ix.search_batch(queries, 10, 10)) == FINGERPRINT_TOP10


@pytest.mark.parametrize("k,ef", [(1, 1), (10, 10), (10, 40), (10, 200)])
def test_oracle_matches_golden_results(orc, golden, k, ef):
    ix = orc.OracleIndex(GOLDEN / "kat_m8.vdx")
    ids, d, c = ix.search_batch(integer_matrix(200, 16, 2), k, ef)
    np.testing.assert_array_equal(ids, golden[f"ids_{k}_{ef}"])
    np.testing.assert_array_equal(d.view(np.uint32), golden[f"dists_{k}_{ef}"].view(np.uint32))
    np.testing.assert_array_equal(c, golden[f"counts_{k}_{ef}"])


def test_oracle_distances_are_bitwise_the_references(orc, golden):
    o = orc.Oracle()
    for a, b, dim, l2, ip in zip(golden["pair_a"], golden["pair_b"], golden["pair_dim"],
                                 golden["pair_l2"], golden["pair_ip"]):
        assert np.float32(o.l2(a[:dim], b[:dim])) == l2, f"l2 dim {dim}"
        assert np.float32(o.ip(a[:dim], b[:dim])) == ip, f"ip dim {dim}"


def test_planted_rounding_mistake_is_caught(orc, golden):
    """With the tail summed the other way, the pinned pairs disagree: the check has teeth."""
    o = orc.Oracle()
    o.L.vo_set_tail_mode(2)
    try:
        mismatches = sum(
            np.float32(o.ip(a[:dim], b[:dim])) != ip
            for a, b, dim, ip in zip(golden["pair_a"], golden["pair_b"], golden["pair_dim"],
                                     golden["pair_ip"]))
    finally:
        o.L.vo_set_tail_mode(0)
    assert mismatches > 0


def test_oracle_bruteforce_matches_golden(orc, golden):
    ids, d, c = orc.Oracle().bruteforce(integer_matrix(1000, 16, 1), integer_matrix(200, 16, 2), 10)
    np.testing.assert_array_equal(ids, golden["bf_ids"])
    np.testing.assert_array_equal(d, golden["bf_dists"])


def test_oracle_bruteforce_known_answers(orc):
    """tests/brute_force_test.cpp:46-73 and :158-175 of the reference."""
    o = orc.Oracle()
    line = np.array([[10.0], [0.0], [7.0], [3.0], [-2.0]], np.float32)
    ids, d, c = o.bruteforce(line, np.array([[2.0]], np.float32), 3)
    assert list(zip(d[0], ids[0])) == [(1.0, 3), (4.0, 1), (16.0, 4)]
    ties = np.array([[4.0], [-4.0], [4.0], [9.0], [-4.0]], np.float32)
    ids, d, c = o.bruteforce(ties, np.array([[0.0]], np.float32), 4)
    assert list(ids[0]) == [0, 1, 2, 4] and list(d[0]) == [16.0] * 4
    ip = np.array([[1, 0], [0, 2], [3, 3]], np.float32)
    ids, d, c = o.bruteforce(ip, np.array([[1, 1]], np.float32), 3, metric=1)
    assert list(zip(d[0], ids[0])) == [(-5.0, 2), (-1.0, 1), (0.0, 0)]
    cos = np.array([[1, 0], [0, 1], [-1, 0]], np.float32)  # stored unit-length
    ids, d, c = o.bruteforce(cos, np.array([[2, 0]], np.float32), 3, metric=2)
    assert list(zip(d[0], ids[0])) == [(0.0, 0), (1.0, 1), (2.0, 2)]


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("dim", [16, 13, 100])
def test_oracle_search_equals_reference(orc, tmp_path, metric, dim):
    """Non-integer data: the restatement's traversal and distances equal the reference's."""
    base = uniform_matrix(1500, dim, 1)
    queries = uniform_matrix(60, dim, 2)
    ref = orc.RefHnsw(dim, metric, 8, 40, 42)
    ref.add(base, threads=1)
    ref.save(tmp_path / "g.vdx")
    ix = orc.OracleIndex(tmp_path / "g.vdx")
    for k, ef in [(1, 1), (10, 10), (10, 40), (10, 200)]:
        a = ref.search_batch(queries, k, ef)
        b = ix.search_batch(queries, k, ef)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
        np.testing.assert_array_equal(a[2], b[2])


def test_distance_known_values(orc):
    """tests/distance_test.cpp:16-59 of the reference."""
    o = orc.Oracle()
    assert o.l2(np.zeros(2), np.array([3.0, 4.0])) == 25.0
    a = np.arange(128, dtype=np.float32)
    b = 127 - a
    assert o.l2(a, b) == float(((a - b).astype(np.int64) ** 2).sum())
    assert o.ip(np.array([1.0, 2, 3]), np.array([4.0, -5, 6])) == 12.0
    assert o.l2(np.zeros(0), np.zeros(0)) == 0.0


def test_traversal_quantizers_match_torch(orc):
    """The oracle's BF16 and E4M3 rounding (which pins the GPU's low-precision traversal) against
    torch's independent CPU conversions, on values spread over 2^-30 .. 2^10 with subnormal E4M3
    inputs, exact ties, +-0 and the saturation edge (torch's E4M3 cast does not saturate, so its
    inputs are clipped to +-448 first)."""
    torch = pytest.importorskip("torch")
    o = orc.Oracle()
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(20000) * np.exp(rng.uniform(-20, 7, 20000))).astype(np.float32)
    edge = np.array([0.0, -0.0, 448, -448, 447.9, 464, 500, -1e9, 2 ** -9, 2 ** -10, 3 * 2 ** -11,
                     1.0625, 1.1875, -1.0625, 2 ** -6 * 1.0625, 2 ** -6 * 1.1875, 3 * 2 ** -10],
                    np.float32)
    x = np.concatenate([x, edge])
    e4m3 = np.array([o.L.vo_e4m3_round(float(v)) for v in x], np.float32)
    want = torch.from_numpy(np.clip(x, -448, 448)).to(torch.float8_e4m3fn).to(torch.float32).numpy()
    np.testing.assert_array_equal(e4m3.view(np.uint32), want.view(np.uint32))
    bf = np.array([o.L.vo_bf16_round(float(v)) for v in x], np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(bf.view(np.uint32), want.view(np.uint32))
    # Whole rows: FP8 with the per-row scale max|x| / 448 (the largest element maps to 448).
    rows = rng.uniform(-3, 3, size=(50, 37)).astype(np.float32)
    q8 = o.quantize_rows(rows, "fp8")
    s = (np.abs(rows).max(axis=1) / np.float32(448)).astype(np.float32)
    codes = torch.from_numpy(np.clip(rows / s[:, None], -448, 448)).to(torch.float8_e4m3fn)
    back = (s[:, None] * codes.to(torch.float32).numpy()).astype(np.float32)
    np.testing.assert_array_equal(q8.view(np.uint32), back.view(np.uint32))
    np.testing.assert_array_equal(o.quantize_rows(rows, "bf16").view(np.uint32),
                                  torch.from_numpy(rows).to(torch.bfloat16).to(torch.float32).numpy().view(np.uint32))
