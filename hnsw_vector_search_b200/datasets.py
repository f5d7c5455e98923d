"""Seeded synthetic workloads.

The reference measures on SIFT1M and GloVe-100, which are not available here; these generators
stand in for them with the same shapes and comparable value distributions (no dataset record is
reproduced). Every generator is deterministic: numpy PCG64 with the seed given, so the base set,
the queries and therefore every graph built from them are reproducible on any machine.

  integer_clusters  1M x 128 (or 10k x 128) L2, SIFT-like: non-negative integers in [0, 255]
                    drawn from a mixture of Gaussian clusters, clipped and rounded (stored as
                    float32). Isotropic sigma (the 10k CPU-runnable case) or per-cluster,
                    per-dimension sigma log-uniform in [2, 30] (the 1M headline case).
  heavy_tailed      1,183,514 x 100 cosine, GloVe-like: Student-t (nu = 3) coordinates times a
                    seeded 100 x 100 mixing matrix with singular values i^-0.7, unit-normalized;
                    queries include a share of exact duplicates of base rows.
  scaled_clusters   N x 96 inner product: a mixture of 4,096 Gaussian clusters whose per-cluster
                    scale is log-normal(0, 0.5), so vector norms vary.
"""

from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _centers(n_clusters: int, dim: int, seed: int, low: float, high: float) -> np.ndarray:
    return _rng(seed).uniform(low, high, size=(n_clusters, dim))


def integer_clusters(rows: int, dim: int, n_clusters: int, seed: int, centers_seed: int,
                     sigma: float | None = None, sigma_range: tuple[float, float] = (2.0, 30.0),
                     chunk: int = 1 << 16) -> np.ndarray:
    """Rows of a Gaussian mixture rounded to integers in [0, 255] (float32).

    The mixture (centers and sigmas) is fixed by `centers_seed`, the rows by `seed`, so base and
    queries drawn with different `seed` come from the same mixture. With `sigma` the clusters are
    isotropic; otherwise each cluster has its own per-dimension sigma, log-uniform in
    `sigma_range`.
    """
    centers = _centers(n_clusters, dim, centers_seed, 0.0, 128.0)
    if sigma is None:
        lo, hi = np.log(sigma_range[0]), np.log(sigma_range[1])
        sigmas = np.exp(_rng(centers_seed + 1).uniform(lo, hi, size=(n_clusters, dim)))
    else:
        sigmas = np.full((n_clusters, dim), float(sigma))
    g = _rng(seed)
    out = np.empty((rows, dim), dtype=np.float32)
    for start in range(0, rows, chunk):
        stop = min(rows, start + chunk)
        which = g.integers(0, n_clusters, size=stop - start)
        x = centers[which] + sigmas[which] * g.standard_normal((stop - start, dim))
        out[start:stop] = np.rint(np.clip(x, 0.0, 255.0))
    return out


def heavy_tailed(rows: int, dim: int, seed: int, mix_seed: int, nu: float = 3.0,
                 decay: float = 0.7, chunk: int = 1 << 16) -> np.ndarray:
    """Unit-norm rows: Student-t(nu) coordinates times a seeded mixing matrix whose singular
    values decay as i^-decay."""
    m = _rng(mix_seed)
    u, _ = np.linalg.qr(m.standard_normal((dim, dim)))
    v, _ = np.linalg.qr(m.standard_normal((dim, dim)))
    s = np.arange(1, dim + 1, dtype=np.float64) ** (-decay)
    mix = (u * s) @ v.T
    g = _rng(seed)
    out = np.empty((rows, dim), dtype=np.float32)
    for start in range(0, rows, chunk):
        stop = min(rows, start + chunk)
        x = g.standard_t(nu, size=(stop - start, dim)) @ mix
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        out[start:stop] = x
    return out


def with_duplicates(queries: np.ndarray, base: np.ndarray, share: float, seed: int) -> np.ndarray:
    """`queries` with a `share` of its rows replaced by exact copies of random base rows."""
    g = _rng(seed)
    q = queries.copy()
    count = int(round(share * len(q)))
    rows = g.choice(len(q), size=count, replace=False)
    q[rows] = base[g.integers(0, len(base), size=count)]
    return q


def scaled_clusters(rows: int, dim: int, n_clusters: int, seed: int, centers_seed: int,
                    chunk: int = 1 << 16) -> np.ndarray:
    """A mixture of isotropic clusters whose scales are log-normal(0, 0.5)."""
    c = _rng(centers_seed)
    centers = c.standard_normal((n_clusters, dim))
    scales = np.exp(c.normal(0.0, 0.5, size=n_clusters))
    g = _rng(seed)
    out = np.empty((rows, dim), dtype=np.float32)
    for start in range(0, rows, chunk):
        stop = min(rows, start + chunk)
        which = g.integers(0, n_clusters, size=stop - start)
        x = (centers[which] + 0.25 * g.standard_normal((stop - start, dim))) * scales[which, None]
        out[start:stop] = x
    return out


def mixed_difficulty(queries: np.ndarray, share: float, noise: float, seed: int) -> np.ndarray:
    """A copy of integer-valued `queries` where a `share` of the rows (chosen with `seed`) get
    Gaussian noise of standard deviation `noise`, clipped to [0, 255] and rounded: queries that
    fall between the clusters need a much longer search than the others, the workload learned
    early termination is for."""
    g = _rng(seed)
    out = queries.copy()
    hard = g.random(len(out)) < share
    out[hard] = np.rint(np.clip(out[hard] + g.normal(0.0, noise, size=(int(hard.sum()), out.shape[1])),
                                0.0, 255.0))
    return out.astype(np.float32)


# The workloads, by name: (base, queries) factories.
def config_small_l2(n_queries: int = 1000):
    """10,000 x 128 L2, 100 isotropic clusters (sigma 12), 1,000 queries."""
    base = integer_clusters(10_000, 128, 100, seed=1, centers_seed=101, sigma=12.0)
    queries = integer_clusters(n_queries, 128, 100, seed=2, centers_seed=101, sigma=12.0)
    return base, queries


def config_sift_like(rows: int = 1_000_000, n_queries: int = 10_000):
    """1M x 128 L2, 1,000 anisotropic clusters, 10,000 held-out queries."""
    base = integer_clusters(rows, 128, 1000, seed=11, centers_seed=111)
    queries = integer_clusters(n_queries, 128, 1000, seed=12, centers_seed=111)
    return base, queries


def config_glove_like(rows: int = 1_183_514, n_queries: int = 10_000):
    """1,183,514 x 100 cosine, heavy-tailed; 2% of the queries duplicate base rows."""
    base = heavy_tailed(rows, 100, seed=31, mix_seed=131)
    queries = heavy_tailed(n_queries, 100, seed=32, mix_seed=131)
    return base, with_duplicates(queries, base, 0.02, seed=33)


def config_scaled_ip(rows: int = 10_000_000, n_queries: int = 10_000):
    """N x 96 inner product, 4,096 clusters with log-normal scales."""
    base = scaled_clusters(rows, 96, 4096, seed=51, centers_seed=151)
    queries = scaled_clusters(n_queries, 96, 4096, seed=52, centers_seed=151)
    return base, queries
