"""vecdex's Python index (`vecdex.Index`, python/bindings.cpp:322-416 of the reference) on the GPU.

Same constructor, methods, properties, input rules, errors and result layout as the reference's
binding, so a caller switches the import and keeps its code:

    from hnsw_vector_search_b200.knn import Index
    index = Index("l2", 128, M=16, ef_construction=200)
    index.add_items(base)                       # the host graph build, as in the reference
    ids, distances = index.knn_query(queries, k=10, ef=64)   # searched on the GPU

knn_query returns int64 ids and float32 distances of shape (n, k), closest first, rows padded
with id -1 and distance inf when fewer than k vectors exist (bindings.cpp:242-289). Inputs must
already be float32, C-contiguous and aligned: they are read in place and never converted
silently; anything else raises the reference's TypeError / ValueError with the same wording.
num_threads is accepted for compatibility: it sets the host threads of add_items; knn_query
always runs on the GPU (the results are the same for any value, as in the reference).

Concurrency, as in the reference: any number of knn_query and save calls at once, add_items
alone (a reader-writer lock); no other thread may modify an input array during a call.
"""

from __future__ import annotations

import sys
import threading

import numpy as np

from . import HnswIndex

DEFAULT_EF = 64  # the reference binding's default search breadth (bindings.cpp:40-43)
_SPACES = ("l2", "ip", "cosine")


def _positive(value: int, name: str) -> int:
    if not isinstance(value, (int, np.integer)) or isinstance(value, bool):
        raise TypeError(f"{name} must be an integer, got {type(value).__name__}")
    if value < 1:
        raise ValueError(f"{name} must be positive, got {value}")
    return int(value)


def _threads(value: int) -> int:
    if value < 0:
        raise ValueError(
            f"num_threads must be positive, or 0 for one per hardware thread, got {value}")
    return int(value)


def _rows(data, dim: int, method: str) -> np.ndarray:
    """The caller's float32 rows, in place: a 2-D (n, dim) array or a 1-D (dim,) vector."""
    try:
        memoryview(data)
    except TypeError:
        raise TypeError(f"{method}: data must support the buffer protocol (a NumPy array), "
                        f"got {type(data).__name__}") from None
    arr = np.asarray(data)
    if arr.ndim not in (1, 2):
        raise ValueError(f"{method}: data must be 1-D (one vector) or 2-D (one vector per row), "
                         f"got {arr.ndim}-D")
    native = "<" if sys.byteorder == "little" else ">"
    if arr.dtype.kind != "f" or arr.dtype.itemsize != 4 or arr.dtype.byteorder not in ("=", "|", native):
        raise TypeError(f"{method}: data must be float32, got {arr.dtype}; "
                        "data.astype(np.float32) converts it (a copy)")
    if arr.shape[-1] != dim:
        raise ValueError(f"{method}: vectors have dimension {arr.shape[-1]}, the index has {dim}")
    if arr.size and not arr.flags.c_contiguous:
        raise ValueError(f"{method}: data must be C-contiguous; np.ascontiguousarray(data) makes "
                         "a contiguous copy")
    if arr.ctypes.data % 4 != 0:
        raise ValueError(f"{method}: data is not aligned for float32; data.copy() makes an "
                         "aligned copy")
    return arr.reshape(1, dim) if arr.ndim == 1 else arr


class _ReadWriteLock:
    """Many readers or one writer."""

    def __init__(self):
        self._cond = threading.Condition()
        self._readers = 0
        self._writer = False

    def read(self):
        lock = self

        class _Read:
            def __enter__(self_):
                with lock._cond:
                    while lock._writer:
                        lock._cond.wait()
                    lock._readers += 1

            def __exit__(self_, *exc):
                with lock._cond:
                    lock._readers -= 1
                    lock._cond.notify_all()
        return _Read()

    def write(self):
        lock = self

        class _Write:
            def __enter__(self_):
                with lock._cond:
                    while lock._writer or lock._readers:
                        lock._cond.wait()
                    lock._writer = True

            def __exit__(self_, *exc):
                with lock._cond:
                    lock._writer = False
                    lock._cond.notify_all()
        return _Write()


class Index:
    """Approximate k-nearest-neighbor search over float32 vectors (an HNSW graph), searched on
    the GPU. space: 'l2' (squared Euclidean), 'ip' (1 - inner product) or 'cosine'
    (1 - cosine similarity; vectors are normalized when stored)."""

    def __init__(self, space: str, dim: int, M: int = 16, ef_construction: int = 200,
                 seed: int = 42, *, device: int = 0, _index: HnswIndex | None = None):
        if space not in _SPACES:
            raise ValueError(f"space must be 'l2', 'ip' or 'cosine', got '{space}'")
        if isinstance(seed, bool) or not isinstance(seed, (int, np.integer)) or seed < 0 or seed >= 2 ** 64:
            raise TypeError("seed must be an integer in [0, 2**64)")
        self._device = int(device)
        self._ef = DEFAULT_EF
        self._lock = _ReadWriteLock()
        if _index is not None:
            self._index = _index
            return
        self._index = HnswIndex(_positive(dim, "dim"), space, M=_positive(M, "M"),
                                ef_construction=_positive(ef_construction, "ef_construction"),
                                seed=int(seed))

    # --- properties ---------------------------------------------------------------------------
    @property
    def dim(self) -> int:
        return self._index.dim

    @property
    def space(self) -> str:
        return _SPACES[self._index.info()["metric"]]

    @property
    def M(self) -> int:  # noqa: N802 (the reference's name)
        return self._index.info()["M"]

    @property
    def ef_construction(self) -> int:
        return self._index.info()["ef_construction"]

    @property
    def ef(self) -> int:
        """knn_query's search breadth when its ef argument is None (default 64)."""
        return self._ef

    @ef.setter
    def ef(self, value: int) -> None:
        self._ef = _positive(value, "ef")

    def set_ef(self, ef: int) -> None:
        self.ef = ef

    def __len__(self) -> int:
        with self._lock.read():
            return len(self._index)

    def memory_bytes(self) -> int:
        with self._lock.read():
            return self._index.info()["memory_bytes"]

    def __repr__(self) -> str:
        return (f"<hnsw_vector_search_b200.Index space='{self.space}' dim={self.dim} M={self.M} "
                f"ef_construction={self.ef_construction} ef={self._ef} len={len(self)}>")

    # --- building, saving ---------------------------------------------------------------------
    def add_items(self, data, *, num_threads: int = 1) -> np.ndarray:
        """Adds vectors (host graph build, as in the reference) and returns their consecutive
        int64 ids. The whole batch is checked before any of it is stored."""
        rows = _rows(data, self.dim, "add_items")
        threads = _threads(num_threads)
        with self._lock.write():
            first = len(self._index)
            if len(rows):
                self._index.add(rows, num_threads=threads)
        return np.arange(first, first + len(rows), dtype=np.int64)

    def save(self, path) -> None:
        with self._lock.read():
            self._index.save(path)

    @classmethod
    def load(cls, path, *, device: int = 0) -> "Index":
        """Reads an index written by save (the reference's format); ef starts at 64."""
        index = HnswIndex.load(path)
        return cls(_SPACES[index.info()["metric"]], index.dim, _index=index, device=device)

    # --- search -------------------------------------------------------------------------------
    def knn_query(self, data, k: int = 1, ef: int | None = None, *, num_threads: int = 1):
        """(ids int64 [n, k], distances float32 [n, k]), closest first; -1 / inf padding."""
        queries = _rows(data, self.dim, "knn_query")
        want = _positive(k, "k")
        breadth = self._ef if ef is None else _positive(ef, "ef")
        _threads(num_threads)
        with self._lock.read():
            ids32, dists, _ = self._index.search_batch(queries, want, breadth, device=self._device)
        ids = ids32.astype(np.int64)
        ids[ids32 == 0xFFFFFFFF] = -1
        return ids, np.ascontiguousarray(dists, dtype=np.float32)
