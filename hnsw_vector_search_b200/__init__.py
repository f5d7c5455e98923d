"""B200 batched query path for vecdex HNSW indexes, from Python.

A thin ctypes layer over the C ABI in include/vdx_b200.h (libvdx_b200.so, built in-tree by
`python -m hnsw_vector_search_b200.build`). HnswIndex and BruteForceIndex mirror the reference's
C++ API (include/vecdex/hnsw.hpp, include/vecdex/brute_force.hpp): same constructor arguments,
same methods, same errors (ValueError for the reference's std::invalid_argument, OverflowError
for std::length_error, OSError for save/load failures). Searches run on the GPU only; if the
native library is missing, importing the classes' first use raises instead of falling back.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIBRARY_PATH = _PKG / "libvdx_b200.so"

_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_P = ctypes.c_void_p
_F = ctypes.c_float

METRICS = {"l2": 0, "ip": 1, "cosine": 2}
PRECISIONS = {"fp32": 0, "bf16": 1, "fp8": 2}
NO_ID = 0xFFFFFFFF
STAT_NAMES = ["queries", "expansions", "dist_layer0", "dist_upper", "link_bytes", "row_bytes",
              "rerank_bytes", "duplicates", "prefetch_hits", "learned_stops"]


class _IndexInfo(ctypes.Structure):
    _fields_ = [("size", _U64), ("dim", _U64), ("M", _U64), ("ef_construction", _U64),
                ("seed", _U64), ("max_level", _U64), ("entry_point", _U64),
                ("memory_bytes", _U64), ("metric", _U32)]


class _PlanTiming(ctypes.Structure):
    _fields_ = [("ef_class", _U32), ("warps_per_block", _I32), ("rows_per_round", _U32), ("hash_slots", _U32),
                ("result_capacity", _U32), ("ms", _F), ("global_slots", _U32)]


class _GraphReport(ctypes.Structure):
    _fields_ = [("violations", _U64), ("reachable", _U64), ("max_level", _U64),
                ("mean_degree0", ctypes.c_double)]


class SearchOptions(ctypes.Structure):
    """vdx_search_options: traversal precision, FP32 re-rank width, learned stop, device."""
    _fields_ = [("precision", _U32), ("rerank", _U32), ("learned_stop", _U32),
                ("stop_threshold", _F), ("device", _I32), ("stop_gate", _U32)]


_lib = None


def lib() -> ctypes.CDLL:
    """The native library, loaded once. Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise RuntimeError(f"{LIBRARY_PATH} is missing: run `python -m hnsw_vector_search_b200.build`")
    L = ctypes.CDLL(str(LIBRARY_PATH))
    sigs = {
        "vdx_last_error": (ctypes.c_char_p, []),
        "vdx_version": (ctypes.c_char_p, []),
        "vdx_device_count": (ctypes.c_int, []),
        "vdx_index_create": (ctypes.c_int, [_U64, _U32, _U64, _U64, _U64, ctypes.POINTER(_P)]),
        "vdx_index_free": (None, [_P]),
        "vdx_index_add": (ctypes.c_int, [_P, _P, _U64, _U64, _U64]),
        "vdx_index_add_one": (ctypes.c_int, [_P, _P, _U64, ctypes.POINTER(_U32)]),
        "vdx_index_add_gpu": (ctypes.c_int, [_P, _P, _U64, _U64, _I32]),
        "vdx_index_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
        "vdx_index_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
        "vdx_index_save_device_image": (ctypes.c_int, [_P, ctypes.c_char_p]),
        "vdx_index_load_device_image": (ctypes.c_int, [_P, ctypes.c_char_p, _I32]),
        "vdx_index_graph_hash": (ctypes.c_int, [_P, ctypes.POINTER(_U64)]),
        "vdx_index_info_get": (ctypes.c_int, [_P, ctypes.POINTER(_IndexInfo)]),
        "vdx_index_inspect": (ctypes.c_int, [_P, ctypes.POINTER(_GraphReport), ctypes.c_char_p, _U64]),
        "vdx_search_batch": (ctypes.c_int, [_P, _P, _U64, _U64, _U64, _U64, _P, _P, _P,
                                            ctypes.POINTER(SearchOptions)]),
        "vdx_search": (ctypes.c_int, [_P, _P, _U64, _U64, _U64, _P, _P, ctypes.POINTER(_U32)]),
        "vdx_last_stats": (ctypes.c_int, [_P, _U64]),
        "vdx_index_upload": (ctypes.c_int, [_P, _I32, _U32]),
        "vdx_work_words": (_U64, []),
        "vdx_search_batch_device": (ctypes.c_int, [_P, _P, _U64, _U64, _P, _P, _U32, _U32, _U32,
                                                   _P, _P, _P, _P, ctypes.POINTER(SearchOptions),
                                                   _P]),
        "vdx_bf_create": (ctypes.c_int, [_U64, _U32, ctypes.POINTER(_P)]),
        "vdx_bf_free": (None, [_P]),
        "vdx_bf_add": (ctypes.c_int, [_P, _P, _U64, _U64]),
        "vdx_bf_size": (_U64, [_P]),
        "vdx_bf_search_batch": (ctypes.c_int, [_P, _P, _U64, _U64, _U64, _U32, _P, _P, _P]),
        "vdx_bf_search_batch_device": (ctypes.c_int, [_P, _P, _U64, _U64, _U64, _U32, _P, _P, _P,
                                                      _P, _P]),
        "vdx_batcher_create": (ctypes.c_int, [_P, _I32, _U32, _U32, _U32, _U32, ctypes.POINTER(_P)]),
        "vdx_batcher_free": (None, [_P]),
        "vdx_batcher_run": (ctypes.c_int, [_P, _P, _U64, _P, _P, _P, _P, _P]),
        "vdx_batcher_autotune": (ctypes.c_int, [_P, _P, _U64, _P, _P, _P, _U64, ctypes.POINTER(_U64)]),
        "vdx_batcher_submit": (ctypes.c_int, [_P, _P, _U64, _P, _P]),
        "vdx_batcher_wait": (ctypes.c_int, [_P, _P, _P, _P]),
        "vdx_host_l2": (_F, [_P, _P, _U64]),
        "vdx_host_ip": (_F, [_P, _P, _U64]),
        "vdx_xxh64": (_U64, [_P, _U64, _U64]),
        "vdx_testing_set_tc_wait_ns": (None, [_U64]),
        "vdx_search_kernels_last": (_U32, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class DeviceTimeout(RuntimeError):
    """VDX_ERR_DEVICE_TIMEOUT: a bounded device wait gave up; the kernel released what it held."""


class DeviceBounds(RuntimeError):
    """VDX_ERR_DEVICE_BOUNDS: a kernel met an out-of-range link id in the device graph."""


def _raise(status: int) -> None:
    if status == 0:
        return
    msg = lib().vdx_last_error().decode()
    if status == 1:
        raise ValueError(msg)
    if status == 2:
        raise OverflowError(msg)
    if status == 3:
        raise OSError(msg)
    if status == 6:
        raise DeviceTimeout(msg)
    if status == 7:
        raise DeviceBounds(msg)
    raise RuntimeError(msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _rows(data, dim: int) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
    if a.ndim == 1:
        a = a.reshape(1, -1) if a.size else a.reshape(0, dim)
    return a


def _options(precision="fp32", rerank=0, learned_stop=False, stop_threshold=0.5, device=0,
             stop_gate=0):
    """rerank: 0 = 4k candidates re-scored in FP32 (BF16 / FP8), "none" = no re-rank.
    stop_gate: the learned stop consults its network only once the k-th distance has been
    unchanged for this many expansions in a row (0: at every checkpoint)."""
    rr = 0xFFFFFFFF if rerank == "none" else int(rerank)
    return SearchOptions(PRECISIONS[precision] if isinstance(precision, str) else int(precision),
                         rr, 1 if learned_stop else 0, float(stop_threshold), int(device),
                         int(stop_gate))


class HnswIndex:
    """The reference's HnswIndex (include/vecdex/hnsw.hpp:63-123); searches run on the GPU."""

    def __init__(self, dim: int, metric: str | int = "l2", M: int = 16,
                 ef_construction: int = 200, seed: int = 42, *, _handle=None):
        self._dim = None
        if _handle is not None:
            self._h = _handle
            return
        h = _P()
        m = METRICS[metric] if isinstance(metric, str) else int(metric)
        if dim < 0 or M < 0 or ef_construction < 0:
            raise ValueError("HnswIndex: negative parameter")
        _raise(lib().vdx_index_create(dim, m, M, ef_construction, seed, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.vdx_index_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        i = _IndexInfo()
        _raise(lib().vdx_index_info_get(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in _IndexInfo._fields_}

    @property
    def dim(self) -> int:
        # Fixed for the index's lifetime; info() also sums memory_bytes() over every node, far
        # too slow to run on each search call.
        if self._dim is None:
            self._dim = int(self.info()["dim"])
        return self._dim

    def __len__(self) -> int:
        return self.info()["size"]

    def add(self, rows, num_threads: int = 1, *, device: int | None = None) -> None:
        """The reference's add (num_threads host threads), or with `device` the batched GPU
        build (HnswIndex::add_gpu)."""
        d = self.dim
        a = _rows(rows, d)
        cols = a.shape[1] if a.ndim == 2 else d
        if device is not None:
            _raise(lib().vdx_index_add_gpu(self._h, _ptr(a), a.shape[0], cols, int(device)))
            return
        _raise(lib().vdx_index_add(self._h, _ptr(a), a.shape[0], cols, num_threads))

    def add_one(self, vector) -> int:
        v = np.ascontiguousarray(np.asarray(vector, dtype=np.float32).ravel())
        out = _U32()
        _raise(lib().vdx_index_add_one(self._h, _ptr(v), v.size, ctypes.byref(out)))
        return out.value

    def save(self, path) -> None:
        _raise(lib().vdx_index_save(self._h, os.fsencode(path)))

    def save_device_image(self, path) -> None:
        """Write the FP32 device mirror as a sidecar file (host only): a 4096-byte header naming
        this graph by its XXH64, then the device arrays, each section 4096-byte aligned."""
        _raise(lib().vdx_index_save_device_image(self._h, os.fsencode(path)))

    def load_device_image(self, path, device: int = 0) -> None:
        """Install a sidecar written by save_device_image as the FP32 mirror on `device`, one
        copy per section; raises OSError if it belongs to another graph."""
        _raise(lib().vdx_index_load_device_image(self._h, os.fsencode(path), device))

    def graph_hash(self) -> int:
        """XXH64 of the vectors, levels, layer-0 and upper blocks (the device image's key)."""
        out = _U64()
        _raise(lib().vdx_index_graph_hash(self._h, ctypes.byref(out)))
        return int(out.value)

    @classmethod
    def load(cls, path) -> "HnswIndex":
        h = _P()
        _raise(lib().vdx_index_load(os.fsencode(path), ctypes.byref(h)))
        return cls(0, _handle=h)

    def inspect(self) -> dict:
        r = _GraphReport()
        buf = ctypes.create_string_buffer(512)
        _raise(lib().vdx_index_inspect(self._h, ctypes.byref(r), buf, 512))
        return {"violations": r.violations, "reachable": r.reachable, "max_level": r.max_level,
                "mean_degree0": r.mean_degree0, "first_violation": buf.value.decode()}

    def upload(self, device: int = 0, precision: str = "fp32") -> None:
        _raise(lib().vdx_index_upload(self._h, device, PRECISIONS[precision]))

    def search_batch(self, queries, k: int, ef: int, *, out=None, **options):
        """(ids uint32 [nq, k], distances float32 [nq, k], counts uint32 [nq]); rows shorter
        than k are padded with 0xFFFFFFFF / +inf. `out` = (ids, distances, counts) arrays of
        those dtypes and shapes, C-contiguous, to fill instead of new ones; page-locked ones
        (e.g. from torch's pin_memory) are written by the GPU in place."""
        q = _rows(queries, self.dim)
        nq = q.shape[0]
        dim = q.shape[1] if q.ndim == 2 else self.dim
        kk = max(int(k), 0)
        if out is None:
            ids = np.empty((nq, kk), np.uint32)
            dists = np.empty((nq, kk), np.float32)
            counts = np.empty(nq, np.uint32)
        else:
            ids, dists, counts = out
            for a, dt, shape, name in ((ids, np.uint32, (nq, kk), "ids"), (dists, np.float32, (nq, kk), "distances"),
                                       (counts, np.uint32, (nq,), "counts")):
                if not isinstance(a, np.ndarray) or a.dtype != dt or a.shape != shape or not a.flags.c_contiguous \
                        or not a.flags.writeable:
                    raise ValueError(f"search_batch: out {name} must be a writable C-contiguous "
                                     f"{np.dtype(dt).name} array of shape {shape}")
        if k < 0 or ef < 0:
            raise ValueError("HnswIndex::search_batch: k and ef must be non-negative")
        opts = _options(**options)
        _raise(lib().vdx_search_batch(self._h, _ptr(q), nq, dim, kk, ef, _ptr(ids), _ptr(dists),
                                      _ptr(counts), ctypes.byref(opts)))
        return ids, dists, counts

    def search(self, query, k: int, ef: int):
        """[(distance, id), ...] closest first, like HnswIndex::search."""
        q = np.ascontiguousarray(np.asarray(query, dtype=np.float32).ravel())
        ids = np.empty(max(k, 0), np.uint32)
        d = np.empty(max(k, 0), np.float32)
        c = _U32()
        if k < 0 or ef < 0:
            raise ValueError("HnswIndex::search: k and ef must be non-negative")
        _raise(lib().vdx_search(self._h, _ptr(q), q.size, k, ef, _ptr(ids), _ptr(d), ctypes.byref(c)))
        return [(float(d[i]), int(ids[i])) for i in range(c.value)]

    @staticmethod
    def last_stats() -> dict:
        out = np.zeros(16, np.uint64)
        _raise(lib().vdx_last_stats(_ptr(out), 16))
        return {n: int(out[i]) for i, n in enumerate(STAT_NAMES)}

    def search_batch_device(self, queries, k_uniform: int, ef_uniform: int, out_stride: int,
                            ids, dists, counts, work, *, k_per_query=None, ef_per_query=None,
                            stream=0, **options) -> None:
        """Asynchronous device-buffer search (torch CUDA tensors or raw device pointers)."""
        def p(t):
            if t is None:
                return None
            return t if isinstance(t, int) else t.data_ptr()
        nq = queries.shape[0]
        opts = _options(**options)
        _raise(lib().vdx_search_batch_device(
            self._h, p(queries), nq, queries.shape[1], p(k_per_query), p(ef_per_query),
            k_uniform, ef_uniform, out_stride, p(ids), p(dists), p(counts), p(work),
            ctypes.byref(opts), stream))


class Batcher:
    """Uneven batches (any size up to max_queries, per-query k and ef) through one CUDA graph
    captured at construction and replayed per batch. Queries are split into ef classes
    (effective ef <= 64, <= 256, <= 1024, ...) that run as concurrent graph branches, each with
    its own launch plan; `autotune` picks those plans. Row i of a result equals
    HnswIndex.search_batch of query i with its own k and ef.

    The batcher keeps the device graph it was made with: make a new one after adding vectors."""

    def __init__(self, index: HnswIndex, max_queries: int, max_k: int, max_ef: int,
                 precision: str = "fp32", device: int = 0):
        self.index = index
        self.max_k = int(max_k)
        h = _P()
        _raise(lib().vdx_batcher_create(index.handle, device, PRECISIONS[precision], max_queries,
                                        max_k, max_ef, ctypes.byref(h)))
        self._h = h.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vdx_batcher_free(self._h)
            self._h = None

    @staticmethod
    def _per_query(v, nq):
        return np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.uint32), (nq,)))

    def run(self, queries, k, ef):
        """(ids [nq, max_k], distances [nq, max_k], counts [nq]); row i holds k[i] results."""
        q = _rows(queries, self.index.dim)
        nq = q.shape[0]
        kk, ee = self._per_query(k, nq), self._per_query(ef, nq)
        ids = np.empty((nq, self.max_k), np.uint32)
        d = np.empty((nq, self.max_k), np.float32)
        c = np.empty(nq, np.uint32)
        _raise(lib().vdx_batcher_run(self._h, _ptr(q), nq, _ptr(kk), _ptr(ee), _ptr(ids), _ptr(d),
                                     _ptr(c)))
        return ids, d, c

    def submit(self, queries, k, ef) -> None:
        """Starts a batch without waiting; `wait` returns its results. One batch in flight per
        batcher (several batchers keep several in flight)."""
        q = _rows(queries, self.index.dim)
        nq = q.shape[0]
        kk, ee = self._per_query(k, nq), self._per_query(ef, nq)
        _raise(lib().vdx_batcher_submit(self._h, _ptr(q), nq, _ptr(kk), _ptr(ee)))
        self._pending = nq

    def wait(self):
        nq = getattr(self, "_pending", None)
        if nq is None:
            raise ValueError("Batcher.wait: no batch was submitted")
        self._pending = None
        ids = np.empty((nq, self.max_k), np.uint32)
        d = np.empty((nq, self.max_k), np.float32)
        c = np.empty(nq, np.uint32)
        _raise(lib().vdx_batcher_wait(self._h, _ptr(ids), _ptr(d), _ptr(c)))
        return ids, d, c

    def autotune(self, queries, k, ef) -> list[dict]:
        """Times every candidate plan on this batch and keeps the fastest; returns the timings."""
        q = _rows(queries, self.index.dim)
        nq = q.shape[0]
        kk, ee = self._per_query(k, nq), self._per_query(ef, nq)
        out = (_PlanTiming * 64)()
        n = _U64()
        _raise(lib().vdx_batcher_autotune(self._h, _ptr(q), nq, _ptr(kk), _ptr(ee),
                                          ctypes.addressof(out), 64, ctypes.byref(n)))
        return [{f: getattr(out[i], f) for f, _ in _PlanTiming._fields_}
                for i in range(min(n.value, 64))]


class BruteForceIndex:
    """The reference's BruteForceIndex (include/vecdex/brute_force.hpp:21-43) on the GPU."""

    def __init__(self, dim: int, metric: str | int = "l2"):
        h = _P()
        m = METRICS[metric] if isinstance(metric, str) else int(metric)
        _raise(lib().vdx_bf_create(dim, m, ctypes.byref(h)))
        self._h = h
        self._dim = dim

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.vdx_bf_free(h)
            self._h = None

    def __len__(self) -> int:
        return int(lib().vdx_bf_size(self._h))

    def add(self, rows) -> None:
        a = _rows(rows, self._dim)
        _raise(lib().vdx_bf_add(self._h, _ptr(a), a.shape[0], a.shape[1] if a.ndim == 2 else self._dim))

    def search_batch(self, queries, k: int, method: str = "tensor_core"):
        """(ids, distances, counts) of the k closest stored vectors per query. "tensor_core" (the
        default) returns the same ids and distance bits as "exact" (certified candidates from the
        tensor cores, exact fallback per query); "exact" scores every pair on the CUDA cores."""
        q = _rows(queries, self._dim)
        nq = q.shape[0]
        kk = max(int(k), 0)
        ids = np.empty((nq, kk), np.uint32)
        dists = np.empty((nq, kk), np.float32)
        counts = np.empty(nq, np.uint32)
        m = {"exact": 0, "tensor_core": 1}[method]
        _raise(lib().vdx_bf_search_batch(self._h, _ptr(q), nq, q.shape[1] if q.ndim == 2 else self._dim,
                                         kk, m, _ptr(ids), _ptr(dists), _ptr(counts)))
        return ids, dists, counts

    def search_batch_device(self, queries, k: int, ids, dists, counts, work, method="tensor_core",
                            stream=0) -> None:
        """Asynchronous device-buffer brute force (torch CUDA tensors)."""
        m = {"exact": 0, "tensor_core": 1}[method]
        _raise(lib().vdx_bf_search_batch_device(
            self._h, queries.data_ptr(), queries.shape[0], queries.shape[1], k, m,
            ids.data_ptr(), dists.data_ptr(), counts.data_ptr(), work.data_ptr(), stream))

    @staticmethod
    def last_uncertified() -> int:
        out = np.zeros(16, np.uint64)
        _raise(lib().vdx_last_stats(_ptr(out), 16))
        return int(out[12])

    def search(self, query, k: int):
        ids, d, c = self.search_batch(np.asarray(query, np.float32).reshape(1, -1), k)
        return [(float(d[0, i]), int(ids[0, i])) for i in range(int(c[0]))]


def host_l2(a, b) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(lib().vdx_host_l2(_ptr(a), _ptr(b), a.size))


def host_ip(a, b) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(lib().vdx_host_ip(_ptr(a), _ptr(b), a.size))


def xxh64(data: bytes, seed: int = 0) -> int:
    buf = ctypes.create_string_buffer(data, len(data))
    return int(lib().vdx_xxh64(ctypes.addressof(buf), len(data), seed))


def device_count() -> int:
    return int(lib().vdx_device_count())
