"""Generates the golden fixtures in this directory from the unmodified reference library.

    python tests/golden/make_golden.py      (needs oracle/_ref/libvecdex_ref.so)

  kat_m8.vdx         the graph of the reference's SerialBuildIsUnchanged test
                     (tests/hnsw_parallel_test.cpp:146-169): integer_matrix(1000, 16, seed 1),
                     M = 8, ef_construction = 64, seed 42, serial build, saved by the reference.
  kat_results.npz    the reference's search results on that graph for integer_matrix(200, 16,
                     seed 2) at (k, ef) in {(1, 1), (10, 10), (10, 40), (10, 200)}, plus its exact
                     brute-force top 10 of the same queries, and its distances for a set of
                     random vector pairs at every dim 0..100 and the common embedding sizes.
  tiny.vdx           a 12-node, dim-2, M = 2, ef_construction = 8, seed 42 L2 index (the shape of
                     the reference's corruption-test fixture, docs/FORMAT.md "Example"), built
                     from integer_matrix(12, 2, seed 1); its header equals the documented one.

The reference's published fingerprints for the first two result sets are asserted in the tests,
so these files are checked against the reference's own numbers, not only regenerated from it.
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))

import oracle as o  # noqa: E402

KAT_SETTINGS = [(1, 1), (10, 10), (10, 40), (10, 200)]
DIMS = list(range(0, 101)) + [127, 128, 129, 255, 256, 257, 383, 384, 385, 767, 768, 769, 1023, 1024]


def main():
    orc = o.Oracle()
    base = orc.integer_matrix(1000, 16, 1)
    queries = orc.integer_matrix(200, 16, 2)
    ref = o.RefHnsw(16, 0, 8, 64, 42)
    ref.add(base, threads=1)
    ref.save(HERE / "kat_m8.vdx")
    loaded = o.RefHnsw.load(HERE / "kat_m8.vdx")
    out = {}
    for k, ef in KAT_SETTINGS:
        ids, d, c = loaded.search_batch(queries, k, ef, threads=4)
        out[f"ids_{k}_{ef}"] = ids
        out[f"dists_{k}_{ef}"] = d
        out[f"counts_{k}_{ef}"] = c
    bf = o.RefBruteForce(16, 0)
    bf.add(base)
    ids, d, c = bf.search_batch(queries, 10)
    out["bf_ids"], out["bf_dists"] = ids, d

    # Distances of random pairs at every dim (non-integer values, both signs, varied scale).
    rng = np.random.default_rng(2024)
    r = o.Ref()
    pairs_a, pairs_b, l2s, ips, dims = [], [], [], [], []
    for dim in DIMS:
        a = (rng.standard_normal(dim) * rng.uniform(0.01, 100)).astype(np.float32)
        b = rng.standard_normal(dim).astype(np.float32)
        pairs_a.append(np.pad(a, (0, 1024 - dim)))
        pairs_b.append(np.pad(b, (0, 1024 - dim)))
        l2s.append(r.l2(a, b))
        ips.append(r.ip(a, b))
        dims.append(dim)
    out["pair_a"] = np.array(pairs_a, np.float32)
    out["pair_b"] = np.array(pairs_b, np.float32)
    out["pair_dim"] = np.array(dims, np.int64)
    out["pair_l2"] = np.array(l2s, np.float32)
    out["pair_ip"] = np.array(ips, np.float32)
    out["isa"] = np.array(r.isa())
    np.savez_compressed(HERE / "kat_results.npz", **out)

    tiny = o.RefHnsw(2, 0, 2, 8, 42)
    tiny.add(orc.integer_matrix(12, 2, 1), threads=1)
    tiny.save(HERE / "tiny.vdx")
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
