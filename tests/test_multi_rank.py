"""The multi-GPU host logic on CPU: two gloo ranks (127.0.0.1), local searches by the oracle, the
real exchange and merge of hnsw_vector_search_b200.sharded. The sharded brute force must equal
one search over all rows, ties included; replicas must return every row in batch order."""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def data():
    g = np.random.default_rng(11)
    base = np.rint(g.uniform(0, 8, size=(997, 8))).astype(np.float32)  # integers: many ties
    queries = np.rint(g.uniform(0, 8, size=(40, 8))).astype(np.float32)
    return base, queries


def worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist
    import oracle
    from hnsw_vector_search_b200 import sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        base, queries = data()
        o = oracle.Oracle()
        off, cnt = sharded.shard_rows(len(base), rank, world)
        shard = base[off:off + cnt]
        sb = sharded.ShardedBruteForce(shard, off, local_search=lambda q, k: o.bruteforce(shard, q, k))
        ids, d, c = sb.search_batch(queries, 10)
        np.savez(Path(out_dir) / f"bf_{rank}.npz", ids=ids, d=d, c=c)

        rs = sharded.ReplicaSearch(lambda q, k, ef: o.bruteforce(base, q, k))
        ids, d, c = rs.search_batch(queries, 5, 32)
        np.savez(Path(out_dir) / f"rep_{rank}.npz", ids=ids, d=d, c=c)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_ranks_equal_one_search(tmp_path, orc):
    port = free_port()
    mp.start_processes(worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    base, queries = data()
    o = orc.Oracle()
    want = o.bruteforce(base, queries, 10)
    want5 = o.bruteforce(base, queries, 5)
    for rank in range(2):
        z = np.load(tmp_path / f"bf_{rank}.npz")
        np.testing.assert_array_equal(z["ids"], want[0])
        np.testing.assert_array_equal(z["d"], want[1])
        np.testing.assert_array_equal(z["c"], want[2])
        z = np.load(tmp_path / f"rep_{rank}.npz")
        np.testing.assert_array_equal(z["ids"], want5[0])
        np.testing.assert_array_equal(z["d"], want5[1])


def test_shard_rows_cover_everything():
    from hnsw_vector_search_b200 import sharded
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [sharded.shard_rows(n, r, world) for r in range(world)]
            assert sum(c for _, c in spans) == n
            pos = 0
            for off, c in spans:
                assert off == pos
                pos += c


def test_merge_keeps_the_closer_order():
    from hnsw_vector_search_b200 import sharded
    ids = np.array([[5, 2, 0xFFFFFFFF, 9, 1]], np.uint32)
    d = np.array([[1.0, 1.0, 0.0, 0.5, 3.0]], np.float32)
    i, dd, c = sharded.merge_candidates(ids, d, 3)
    assert list(i[0]) == [9, 2, 5] and list(dd[0]) == [0.5, 1.0, 1.0] and c[0] == 3
