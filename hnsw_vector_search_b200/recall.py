"""Recall of search results against exact ground truth, vectorized over a batch.

Definitions (the reference's measures, include/vecdex/recall.hpp:15-30):
  recall@k            |{first k found ids} ∩ {first k true ids}| / k: order is ignored, a
                      missing result is a miss, a repeated found id counts once;
  threshold recall@k  share of the first k found whose distance is at most the k-th true
                      distance plus tolerance * max(|k-th|, 1).
Missing results are the padding this library writes (id 0xFFFFFFFF / -1, distance +inf), or
rows shorter than k.
"""

from __future__ import annotations

import numpy as np


def _first_k(a, k: int, fill) -> np.ndarray:
    """Rows of `a` (2-D array, or a list of 1-D rows) cut or padded to exactly k columns."""
    if isinstance(a, np.ndarray) and a.ndim == 2:
        out = a[:, :k]
        if out.shape[1] < k:
            out = np.concatenate([out, np.full((len(a), k - out.shape[1]), fill, out.dtype)], 1)
        return out
    rows = [np.asarray(r)[:k] for r in a]
    dtype = np.result_type(*[r.dtype for r in rows]) if rows else np.float64
    out = np.full((len(rows), k), fill, dtype=dtype)
    for i, r in enumerate(rows):
        out[i, :len(r)] = r
    return out


def recall_at_k_per_query(found_ids, truth_ids, k: int) -> np.ndarray:
    """recall@k of every query (float64 array)."""
    if k <= 0:
        raise ValueError("recall_at_k: k must be positive")
    t = np.asarray(truth_ids)
    if t.ndim != 2 or t.shape[1] < k:
        raise ValueError(f"recall_at_k: truth has {t.shape[-1] if t.ndim else 0} ids, fewer than k = {k}")
    t = t[:, :k].astype(np.int64)
    f = _first_k(found_ids, k, -1).astype(np.int64)
    f = np.where((f < 0) | (f == 0xFFFFFFFF), -1, f)
    if len(f) != len(t):
        raise ValueError("recall_at_k: found and truth have different numbers of queries")
    # A true id is a hit when it appears anywhere among the first k found: each true id is
    # counted once, however often it was found.
    hits = (t[:, :, None] == f[:, None, :]).any(axis=2).sum(axis=1)
    return hits / k


def recall_at_k(found_ids, truth_ids, k: int) -> float:
    """Mean recall@k over the queries."""
    return float(recall_at_k_per_query(found_ids, truth_ids, k).mean())


def threshold_recall_at_k(found_dists, kth_true_dists, k: int, tolerance: float = 1e-5) -> float:
    """Mean threshold recall@k; kth_true_dists holds each query's k-th true distance."""
    if k <= 0:
        raise ValueError("threshold_recall_at_k: k must be positive")
    kth = np.asarray(kth_true_dists, np.float32).reshape(-1)
    if not np.all(np.isfinite(kth)) or not np.isfinite(tolerance) or tolerance < 0:
        raise ValueError("threshold_recall_at_k: distance and tolerance must be finite, tolerance >= 0")
    d = _first_k(found_dists, k, np.inf).astype(np.float32)
    limit = kth + np.float32(tolerance) * np.maximum(np.abs(kth), np.float32(1.0))
    return float(((d <= limit[:, None]).sum(axis=1) / k).mean())
