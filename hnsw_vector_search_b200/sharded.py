"""Multi-GPU forms of the batched query path: one process per GPU, torch.distributed for the one
exchange step.

* Exact brute force shards by stored rows. Rank r holds rows [offset_r, offset_r + n_r) of the
  collection, finds each query's k best among them on its GPU, and one all-gather exchanges the
  (distance, global id) candidates (nq x k x 8 bytes per rank); every rank then merges them in the
  reference's `closer` order. The global top k is among the union of the shards' top k, so the
  result equals a single-GPU search over all rows, ties included.
* HNSW search does not shard (a graph per shard is a different graph, with different results),
  so it runs as replicas: each rank searches its own slice of a batch on a full copy of the index,
  and one all-gather returns every row to every rank, in the batch's order.

The local searches are the GPU searches of this package; the exchange works over NCCL (CUDA
tensors) or gloo (CPU tensors, which the tests use).
"""

from __future__ import annotations

import numpy as np


def merge_candidates(ids: np.ndarray, dists: np.ndarray, k: int):
    """Per row, the k best of `ids` / `dists` ([nq, m], id 0xFFFFFFFF = empty) by (distance, id);
    returns (ids [nq, k] uint32, dists [nq, k] float32, counts [nq] uint32)."""
    ids = np.asarray(ids, np.uint32)
    dists = np.asarray(dists, np.float32)
    nq = ids.shape[0]
    out_i = np.full((nq, k), 0xFFFFFFFF, np.uint32)
    out_d = np.full((nq, k), np.inf, np.float32)
    counts = np.zeros(nq, np.uint32)
    for q in range(nq):
        valid = ids[q] != 0xFFFFFFFF
        order = np.lexsort((ids[q][valid], dists[q][valid]))[:k]
        c = len(order)
        out_i[q, :c] = ids[q][valid][order]
        out_d[q, :c] = dists[q][valid][order]
        counts[q] = c
    return out_i, out_d, counts


def exchange_candidates(ids: np.ndarray, dists: np.ndarray, group=None, device=None):
    """All-gathers every rank's [nq, k] candidates; returns ([nq, world * k] ids, dists)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    t_ids = torch.from_numpy(np.ascontiguousarray(ids, np.uint32).view(np.int32))
    t_d = torch.from_numpy(np.ascontiguousarray(dists, np.float32))
    if device is not None:
        t_ids, t_d = t_ids.to(device), t_d.to(device)
    all_ids = [torch.empty_like(t_ids) for _ in range(world)]
    all_d = [torch.empty_like(t_d) for _ in range(world)]
    dist.all_gather(all_ids, t_ids, group=group)
    dist.all_gather(all_d, t_d, group=group)
    cat_i = torch.cat(all_ids, dim=1).cpu().numpy().view(np.uint32)
    cat_d = torch.cat(all_d, dim=1).cpu().numpy()
    return cat_i, cat_d


def shard_rows(n: int, rank: int, world: int) -> tuple[int, int]:
    """[offset, offset + count) of the rows rank `rank` holds: contiguous, sizes differ by <= 1."""
    base, extra = divmod(n, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


class ShardedBruteForce:
    """Exact brute force over a collection whose rows are split across the ranks."""

    def __init__(self, shard: np.ndarray, offset: int, metric: str = "l2", local_search=None,
                 group=None, device=None):
        self.offset = int(offset)
        self.group = group
        self.device = device
        if local_search is None:
            from . import BruteForceIndex
            index = BruteForceIndex(shard.shape[1], metric)
            index.add(shard)
            local_search = lambda q, k: index.search_batch(q, k)  # noqa: E731
        self.local_search = local_search

    def search_batch(self, queries: np.ndarray, k: int):
        ids, d, _ = self.local_search(queries, k)
        ids = np.where(ids != 0xFFFFFFFF, ids.astype(np.uint64) + self.offset, 0xFFFFFFFF).astype(np.uint32)
        all_i, all_d = exchange_candidates(ids, d, self.group, self.device)
        return merge_candidates(all_i, all_d, k)


class ReplicaSearch:
    """HNSW batch search over replicas: rank r searches rows r, r + world, ... of the batch."""

    def __init__(self, local_search, group=None, device=None):
        self.local_search = local_search
        self.group = group
        self.device = device

    def search_batch(self, queries: np.ndarray, k: int, ef: int):
        import torch.distributed as dist
        world = dist.get_world_size(self.group)
        rank = dist.get_rank(self.group)
        nq = len(queries)
        mine = np.arange(rank, nq, world)
        per = (nq + world - 1) // world
        ids = np.full((per, k), 0xFFFFFFFF, np.uint32)
        d = np.full((per, k), np.inf, np.float32)
        if len(mine):
            li, ld, _ = self.local_search(queries[mine], k, ef)
            ids[:len(mine)], d[:len(mine)] = li, ld
        all_i, all_d = exchange_candidates(ids, d, self.group, self.device)
        out_i = np.empty((nq, k), np.uint32)
        out_d = np.empty((nq, k), np.float32)
        for r in range(world):
            rows = np.arange(r, nq, world)
            out_i[rows] = all_i[:len(rows), r * k:(r + 1) * k]
            out_d[rows] = all_d[:len(rows), r * k:(r + 1) * k]
        counts = (out_i != 0xFFFFFFFF).sum(axis=1).astype(np.uint32)
        return out_i, out_d, counts
