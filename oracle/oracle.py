"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: Python access to the two checkers.

  Ref     the unmodified vecdex reference (oracle/_ref/libvecdex_ref.so, compiled from the
          reference's own sources by oracle/Makefile) through ref_shim.cpp's C ABI;
  Oracle  this repository's plain-C restatement of the path (oracle/_build/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libvecdex_ref.so"
ORACLE_LIB = HERE / "_build" / "liboracle.so"

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_F = ctypes.c_float


def ref_root() -> Path:
    """The reference project's checkout: $REF_ROOT, else `reference` beside this repository."""
    return Path(os.environ.get("REF_ROOT", HERE.parent.parent / "reference"))


def build(ref: bool = True) -> None:
    """Compiles the restatement, and the reference when its sources are present."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    root = ref_root()
    if ref and root.joinpath("src").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_ROOT={root}"], check=True)


INTEGRATION_BIN = HERE / "_ref" / "gpu_searcher"


def build_integration() -> bool:
    """Compiles tests/integration/gpu_searcher.cpp (the vecdex-side C++ caller of the C ABI)
    against the reference's headers when they are present; True when the program exists."""
    root = ref_root()
    if root.joinpath("include", "vecdex", "hnsw.hpp").exists() and REF_LIB.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "integration", f"REF_ROOT={root}"], check=True)
    return INTEGRATION_BIN.exists()


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class Ref:
    """The reference library (its public C++ API behind ref_shim.cpp)."""

    _lib = None

    def __init__(self):
        if Ref._lib is None:
            if not REF_LIB.exists():
                raise RuntimeError(f"{REF_LIB} is missing: run `make -C oracle ref`")
            L = ctypes.CDLL(str(REF_LIB))
            L.vref_last_error.restype = ctypes.c_char_p
            L.vref_isa.restype = ctypes.c_char_p
            for n in ("vref_l2", "vref_ip"):
                getattr(L, n).restype = _F
                getattr(L, n).argtypes = [_P, _P, _U64]
            L.vref_hnsw_new.argtypes = [_U64, ctypes.c_int, _U64, _U64, _U64, ctypes.POINTER(_P)]
            L.vref_hnsw_free.argtypes = [_P]
            L.vref_hnsw_add.argtypes = [_P, _P, _U64, _U64, _U64]
            L.vref_hnsw_add_one.argtypes = [_P, _P, _U64, ctypes.POINTER(_U32)]
            L.vref_hnsw_save.argtypes = [_P, ctypes.c_char_p]
            L.vref_hnsw_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(_P)]
            L.vref_hnsw_info.argtypes = [_P] + [ctypes.POINTER(_U64)] * 2 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.POINTER(_U64)] * 2
            L.vref_hnsw_inspect.argtypes = [_P] + [ctypes.POINTER(_U64)] * 3 + [ctypes.POINTER(ctypes.c_double)]
            L.vref_hnsw_search.argtypes = [_P, _P, _U64, _U64, _U64, _P, _P, ctypes.POINTER(_U32)]
            L.vref_hnsw_search_batch.argtypes = [_P, _P, _U64, _U64, _U64, _U64, _U64, _P, _P, _P]
            L.vref_hnsw_time_search_batch.argtypes = [_P, _P, _U64, _U64, _U64, _U64, _U64, _U64, _P]
            L.vref_bf_new.argtypes = [_U64, ctypes.c_int, ctypes.POINTER(_P)]
            L.vref_bf_free.argtypes = [_P]
            L.vref_bf_add.argtypes = [_P, _P, _U64, _U64]
            L.vref_bf_search_batch.argtypes = [_P, _P, _U64, _U64, _U64, _U64, _P, _P, _P]
            Ref._lib = L
        self.L = Ref._lib

    def check(self, rc: int) -> None:
        if rc != 0:
            msg = self.L.vref_last_error().decode()
            raise {-1: ValueError, -2: OverflowError, -3: OSError}.get(rc, RuntimeError)(msg)

    def isa(self) -> str:
        return self.L.vref_isa().decode()

    def l2(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self.L.vref_l2(_p(a), _p(b), a.size))

    def ip(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self.L.vref_ip(_p(a), _p(b), a.size))


class RefHnsw:
    """A reference HnswIndex."""

    def __init__(self, dim=None, metric=0, M=16, ef_construction=200, seed=42, *, handle=None):
        self.ref = Ref()
        if handle is not None:
            self.h = handle
        else:
            self.h = _P()
            self.ref.check(self.ref.L.vref_hnsw_new(dim, metric, M, ef_construction, seed,
                                                    ctypes.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.vref_hnsw_free(self.h)
            self.h = None

    def add(self, rows, threads=1):
        a = np.ascontiguousarray(rows, np.float32)
        self.ref.check(self.ref.L.vref_hnsw_add(self.h, _p(a), a.shape[0], a.shape[1], threads))

    def add_one(self, v) -> int:
        a = np.ascontiguousarray(v, np.float32).ravel()
        out = _U32()
        self.ref.check(self.ref.L.vref_hnsw_add_one(self.h, _p(a), a.size, ctypes.byref(out)))
        return out.value

    def save(self, path):
        self.ref.check(self.ref.L.vref_hnsw_save(self.h, os.fsencode(path)))

    @classmethod
    def load(cls, path) -> "RefHnsw":
        r = Ref()
        h = _P()
        r.check(r.L.vref_hnsw_load(os.fsencode(path), ctypes.byref(h)))
        return cls(handle=h)

    def info(self) -> dict:
        size, dim, M, mem = _U64(), _U64(), _U64(), _U64()
        metric = ctypes.c_int()
        self.ref.L.vref_hnsw_info(self.h, ctypes.byref(size), ctypes.byref(dim),
                                  ctypes.byref(metric), ctypes.byref(M), ctypes.byref(mem))
        return {"size": size.value, "dim": dim.value, "metric": metric.value, "M": M.value,
                "memory_bytes": mem.value}

    def inspect(self) -> dict:
        v, r, m = _U64(), _U64(), _U64()
        d = ctypes.c_double()
        self.ref.check(self.ref.L.vref_hnsw_inspect(self.h, ctypes.byref(v), ctypes.byref(r),
                                                    ctypes.byref(m), ctypes.byref(d)))
        return {"violations": v.value, "reachable": r.value, "max_level": m.value,
                "mean_degree0": d.value}

    def search(self, q, k, ef):
        q = np.ascontiguousarray(q, np.float32).ravel()
        ids = np.empty(k, np.uint32)
        d = np.empty(k, np.float32)
        c = _U32()
        self.ref.check(self.ref.L.vref_hnsw_search(self.h, _p(q), q.size, k, ef, _p(ids), _p(d),
                                                   ctypes.byref(c)))
        return [(float(d[i]), int(ids[i])) for i in range(c.value)]

    def search_batch(self, queries, k, ef, threads=0):
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.uint32)
        d = np.empty((nq, k), np.float32)
        c = np.empty(nq, np.uint32)
        self.ref.check(self.ref.L.vref_hnsw_search_batch(self.h, _p(q), nq, q.shape[1], k, ef,
                                                         threads, _p(ids), _p(d), _p(c)))
        return ids, d, c

    def time_search_batch(self, queries, k, ef, threads, repeats):
        q = np.ascontiguousarray(queries, np.float32)
        out = np.zeros(repeats, np.float64)
        self.ref.check(self.ref.L.vref_hnsw_time_search_batch(
            self.h, _p(q), q.shape[0], q.shape[1], k, ef, threads, repeats, _p(out)))
        return out


class RefBruteForce:
    def __init__(self, dim, metric=0):
        self.ref = Ref()
        self.h = _P()
        self.ref.check(self.ref.L.vref_bf_new(dim, metric, ctypes.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.L.vref_bf_free(self.h)
            self.h = None

    def add(self, rows):
        a = np.ascontiguousarray(rows, np.float32)
        self.ref.check(self.ref.L.vref_bf_add(self.h, _p(a), a.shape[0], a.shape[1]))

    def search_batch(self, queries, k, threads=0):
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.uint32)
        d = np.empty((nq, k), np.float32)
        c = np.empty(nq, np.uint32)
        self.ref.check(self.ref.L.vref_bf_search_batch(self.h, _p(q), nq, q.shape[1], k, threads,
                                                       _p(ids), _p(d), _p(c)))
        return ids, d, c


class Oracle:
    """The plain-C restatement (vdx_oracle.c)."""

    _lib = None

    def __init__(self):
        if Oracle._lib is None:
            if not ORACLE_LIB.exists():
                build(ref=False)
            L = ctypes.CDLL(str(ORACLE_LIB))
            for n in ("vo_l2", "vo_ip"):
                getattr(L, n).restype = _F
                getattr(L, n).argtypes = [_P, _P, _U64]
            L.vo_set_tail_mode.argtypes = [ctypes.c_int]
            L.vo_normalize.argtypes = [_P, _U64]
            L.vo_index_load.restype = _P
            L.vo_index_load.argtypes = [ctypes.c_char_p]
            L.vo_index_free.argtypes = [_P]
            L.vo_search_batch.argtypes = [_P, _P, _U64, _U64, _U64, _P, _P, _P, _P]
            L.vo_bruteforce_batch.argtypes = [_P, _U64, _U64, ctypes.c_int, _P, _U64, _U64, _P, _P, _P]
            L.vo_fingerprint.restype = _U64
            L.vo_fingerprint.argtypes = [_P, _P, _P, _U64, _U64]
            L.vo_integer_matrix.argtypes = [_U64, _U64, _U32, _P]
            L.vo_index_size.restype = _U64
            L.vo_index_size.argtypes = [_P]
            L.vo_index_dim.restype = _U64
            L.vo_index_dim.argtypes = [_P]
            for n in ("vo_bf16_round", "vo_e4m3_round"):
                getattr(L, n).restype = _F
                getattr(L, n).argtypes = [_F]
            L.vo_quantize_rows.argtypes = [ctypes.c_int, _P, _U64, _U64, _P]
            L.vo_index_quantize.argtypes = [_P, ctypes.c_int]
            Oracle._lib = L
        self.L = Oracle._lib

    def l2(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self.L.vo_l2(_p(a), _p(b), a.size))

    def ip(self, a, b) -> float:
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        return float(self.L.vo_ip(_p(a), _p(b), a.size))

    def quantize_rows(self, rows, precision: str) -> np.ndarray:
        """The GPU traversal copy of `rows` as FP32 values: "bf16" (round to nearest even) or
        "fp8" (E4M3 with a per-row FP32 scale max|x| / 448, round to nearest even, saturating)."""
        a = np.ascontiguousarray(rows, np.float32)
        out = np.empty_like(a)
        code = {"fp32": 0, "bf16": 1, "fp8": 2}[precision]
        self.L.vo_quantize_rows(code, _p(a), a.shape[0], a.shape[1], _p(out))
        return out

    def integer_matrix(self, rows, dim, seed) -> np.ndarray:
        out = np.empty((rows, dim), np.float32)
        self.L.vo_integer_matrix(rows, dim, seed, _p(out))
        return out

    def fingerprint(self, ids, dists, counts) -> int:
        ids = np.ascontiguousarray(ids, np.uint32)
        dists = np.ascontiguousarray(dists, np.float32)
        counts = np.ascontiguousarray(counts, np.uint32)
        return int(self.L.vo_fingerprint(_p(ids), _p(dists), _p(counts), ids.shape[0], ids.shape[1]))

    def bruteforce(self, base, queries, k, metric=0):
        """Exact top-k; `base` as the index stores it (normalized under cosine)."""
        b = np.ascontiguousarray(base, np.float32)
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.uint32)
        d = np.empty((nq, k), np.float32)
        c = np.empty(nq, np.uint32)
        self.L.vo_bruteforce_batch(_p(b), b.shape[0], b.shape[1], metric, _p(q), nq, k, _p(ids),
                                   _p(d), _p(c))
        return ids, d, c


class OracleIndex:
    """An index file loaded by the restatement (valid files only)."""

    def __init__(self, path):
        self.o = Oracle()
        self.h = self.o.L.vo_index_load(os.fsencode(path))
        if not self.h:
            raise OSError(f"oracle could not read {path}")

    def __del__(self):
        if getattr(self, "h", None):
            self.o.L.vo_index_free(self.h)
            self.h = None

    def quantize(self, precision: str) -> None:
        """Replaces the stored vectors by their traversal copy ("bf16" or "fp8"), so that
        searches run the GPU's low-precision traversal."""
        self.o.L.vo_index_quantize(self.h, {"bf16": 1, "fp8": 2}[precision])

    def search_batch(self, queries, k, ef, stats=False):
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.uint32)
        d = np.empty((nq, k), np.float32)
        c = np.empty(nq, np.uint32)
        st = np.zeros((nq, 5), np.uint64) if stats else None
        self.o.L.vo_search_batch(self.h, _p(q), nq, k, ef, _p(ids), _p(d), _p(c),
                                 _p(st) if stats else None)
        return (ids, d, c, st) if stats else (ids, d, c)
