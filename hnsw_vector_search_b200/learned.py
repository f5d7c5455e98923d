"""Learned early termination for the GPU HNSW search.

A small network (12 -> 64 -> 64 -> 1, ReLU, sigmoid; bfloat16 weights, FP32 accumulation)
reads a query's search state every 8 expansions and stops the layer-0 beam once it predicts the
top k has converged; ef stays the hard cap, so the plain ef-bounded search is the fallback.

Pipeline (all heavy work on the GPU, through the C ABI):
  1. traces   plain search of training queries at the ef cap the model will run under; every 8
              expansions the 12 features and how many of the current top k are true neighbors
              (exact brute force is the judge), and the final count;
  2. labels   a checkpoint is "converged" when its hit count already equals the final one:
              stopping there would lose nothing against searching on to the cap;
  3. train    vdx_mlp_train: this library's forward / backward / Adam kernels;
  4. calibrate  the stop threshold is the smallest one whose recall on held-out queries meets
              the target at the chosen ef cap.

Model files are .npz with a format version.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _P, _U32, _U64, _raise, _ptr, lib
from .recall import recall_at_k

FEATURES = 12
PARAMS = 5057
MODEL_VERSION = 4


def _bind():
    L = lib()
    if getattr(L, "_learned_bound", False):
        return L
    f = ctypes.c_float
    L.vdx_index_set_stop_model.restype = ctypes.c_int
    L.vdx_index_set_stop_model.argtypes = [_P, _P, _P, _P, _P]
    L.vdx_stop_trace.restype = ctypes.c_int
    L.vdx_stop_trace.argtypes = [_P, _P, _U64, _U64, _P, _U64, _U64, _U64, _P, _U64, _P, _P, _P, _P,
                                 ctypes.c_int32]
    L.vdx_mlp_train.restype = ctypes.c_int
    L.vdx_mlp_train.argtypes = [_P, _P, _U64, _U32, _U64, f, _U64, _P, _P, _P, _P]
    L.vdx_mlp_gradient.restype = ctypes.c_int
    L.vdx_mlp_gradient.argtypes = [_P, _P, _U64, _P, _P, _P]
    L.vdx_mlp_probabilities.restype = ctypes.c_int
    L.vdx_mlp_probabilities.argtypes = [_P, _U64, _P, _P, _P, _P]
    L._learned_bound = True
    return L


@dataclass
class StopModel:
    weights: np.ndarray   # [5057] float32
    mean: np.ndarray      # [12]
    inv_std: np.ndarray   # [12]
    proj: np.ndarray      # [4, dim]
    threshold: float = 0.5
    ef_cap: int = 128
    gate: int = 0         # consult the network only after this many unchanged expansions

    def save(self, path) -> None:
        np.savez(path, version=MODEL_VERSION, weights=self.weights, mean=self.mean,
                 inv_std=self.inv_std, proj=self.proj, threshold=self.threshold, ef_cap=self.ef_cap,
                 gate=self.gate)

    @classmethod
    def load(cls, path) -> "StopModel":
        z = np.load(path)
        if int(z["version"]) != MODEL_VERSION:
            raise ValueError(f"{path}: stop model version {int(z['version'])} is not supported")
        return cls(z["weights"].astype(np.float32), z["mean"].astype(np.float32),
                   z["inv_std"].astype(np.float32), z["proj"].astype(np.float32),
                   float(z["threshold"]), int(z["ef_cap"]), int(z["gate"]))


def random_projections(dim: int, seed: int = 404) -> np.ndarray:
    """Four seeded unit directions: features 8..11 are the query's coordinates along them."""
    g = np.random.Generator(np.random.PCG64(seed))
    p = g.standard_normal((4, dim))
    return (p / np.linalg.norm(p, axis=1, keepdims=True)).astype(np.float32)


def traces(index, queries: np.ndarray, truth: np.ndarray, k: int = 10, ef: int = 512,
           proj: np.ndarray | None = None, max_points: int | None = None, device: int = 0):
    """Checkpoint features and hit counts of the plain search (see the module docstring)."""
    L = _bind()
    q = np.ascontiguousarray(queries, np.float32)
    t = np.ascontiguousarray(truth[:, :k], np.uint32)
    nq, dim = q.shape
    proj = random_projections(dim) if proj is None else np.ascontiguousarray(proj, np.float32)
    mp = max_points or (ef // 8 + 64)
    feats = np.zeros((nq, mp, FEATURES), np.float32)
    hits = np.zeros((nq, mp), np.uint8)
    points = np.zeros(nq, np.uint32)
    final = np.zeros(nq, np.uint8)
    _raise(L.vdx_stop_trace(index.handle, _ptr(q), nq, dim, _ptr(t), k, k, ef, _ptr(proj), mp,
                            _ptr(feats), _ptr(hits), _ptr(points), _ptr(final), device))
    return {"features": feats, "hits": hits, "points": points, "final": final, "proj": proj}


def training_set(tr: dict, max_checkpoint: int | None = None):
    """(x [N, 12], y [N]): every recorded checkpoint, labeled converged when its hits equal the
    final hits."""
    xs, ys = [], []
    pts = tr["points"]
    for qi in range(len(pts)):
        n = int(pts[qi]) if max_checkpoint is None else min(int(pts[qi]), max_checkpoint)
        if n == 0:
            continue
        xs.append(tr["features"][qi, :n])
        ys.append((tr["hits"][qi, :n] >= tr["final"][qi]).astype(np.float32))
    return np.concatenate(xs).astype(np.float32), np.concatenate(ys).astype(np.float32)


def train(x: np.ndarray, y: np.ndarray, proj: np.ndarray, epochs: int = 8, batch: int = 4096,
          lr: float = 1e-3, seed: int = 7):
    """Trains on the GPU with this library's kernels; returns (StopModel, loss per epoch)."""
    L = _bind()
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.zeros(PARAMS, np.float32)
    mean = np.zeros(FEATURES, np.float32)
    inv = np.zeros(FEATURES, np.float32)
    losses = np.zeros(epochs, np.float32)
    _raise(L.vdx_mlp_train(_ptr(x), _ptr(y), len(x), epochs, batch, lr, seed, _ptr(w), _ptr(mean),
                           _ptr(inv), _ptr(losses)))
    return StopModel(w, mean, inv, np.ascontiguousarray(proj, np.float32)), losses


def gradient(x_std: np.ndarray, y: np.ndarray, weights: np.ndarray):
    """GPU gradient of the mean loss over standardized features (for checks)."""
    L = _bind()
    x = np.ascontiguousarray(x_std, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(weights, np.float32)
    g = np.zeros(PARAMS, np.float32)
    loss = ctypes.c_float()
    _raise(L.vdx_mlp_gradient(_ptr(x), _ptr(y), len(x), _ptr(w), _ptr(g), ctypes.byref(loss)))
    return float(loss.value), g


def probabilities(model: StopModel, x: np.ndarray) -> np.ndarray:
    L = _bind()
    x = np.ascontiguousarray(x, np.float32)
    p = np.zeros(len(x), np.float32)
    _raise(L.vdx_mlp_probabilities(_ptr(x), len(x), _ptr(model.weights), _ptr(model.mean),
                                   _ptr(model.inv_std), _ptr(p)))
    return p


def attach(index, model: StopModel) -> None:
    L = _bind()
    _raise(L.vdx_index_set_stop_model(index.handle, _ptr(model.weights), _ptr(model.mean),
                                      _ptr(model.inv_std), _ptr(np.ascontiguousarray(model.proj))))


def recall(ids: np.ndarray, truth: np.ndarray, k: int) -> float:
    return recall_at_k(ids, truth, k)


def calibrate(index, model: StopModel, queries: np.ndarray, truth: np.ndarray, k: int,
              target: float, ef_cap: int, thresholds=None, **options) -> tuple[float, float]:
    """The smallest threshold (fastest stopping) whose recall@k on `queries` meets `target` at
    ef cap `ef_cap`; returns (threshold, recall). Falls back to the largest candidate."""
    attach(index, model)
    cands = thresholds if thresholds is not None else [0.05, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7,
                                                       0.8, 0.85, 0.9, 0.93, 0.95, 0.97, 0.98,
                                                       0.99, 0.995]
    best = None
    for t in sorted(cands):
        ids, _, _ = index.search_batch(queries, k, ef_cap, learned_stop=True, stop_threshold=t,
                                       **options)
        r = recall(ids, truth, k)
        if r >= target:
            best = (t, r)
            break
        best = (t, r)
    model.threshold, model.ef_cap = best[0], ef_cap
    model.gate = int(options.get("stop_gate", 0))
    return best
