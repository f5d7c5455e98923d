"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: the FP64 CPU restatement of the learned-termination
network, the checker for the GPU training kernels (hnsw_vector_search_b200/csrc/mlp.cu).

The network has no counterpart in the reference; this restatement follows the library's own
specification: 12 standardized features -> 64 ReLU -> 64 ReLU -> 1 logit; parameters, in order,
W1 [64][12], b1 [64], W2 [64][64], b2 [64], W3 [64], b3 (5,057); weights (not biases) rounded to
bfloat16 (nearest even) before use; loss = mean binary cross-entropy with logits. Gradients are
with respect to the rounded weights. Computed in float64; finite differences pin it
(tests/test_learned.py).
"""

from __future__ import annotations

import numpy as np

F, H = 12, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
N_PARAMS = OFF_B3 + 1


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 values rounded to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def rounded(w: np.ndarray) -> np.ndarray:
    q = np.array(w, np.float32)
    for lo, hi in ((OFF_W1, OFF_B1), (OFF_W2, OFF_B2), (OFF_W3, OFF_B3)):
        q[lo:hi] = bf16_round(q[lo:hi])
    return q


def unpack(w: np.ndarray):
    w = np.asarray(w, np.float64)
    return (w[OFF_W1:OFF_B1].reshape(H, F), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(H, H),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def forward(x: np.ndarray, wq: np.ndarray):
    W1, b1, W2, b2, W3, b3 = unpack(wq)
    x = np.asarray(x, np.float64)
    a = np.maximum(x @ W1.T + b1, 0.0)
    z = np.maximum(a @ W2.T + b2, 0.0)
    logit = z @ W3 + b3
    return a, z, logit


def loss_and_grad(x: np.ndarray, y: np.ndarray, w: np.ndarray):
    """Mean BCE-with-logits loss and its gradient with respect to the rounded weights."""
    wq = rounded(w)
    W1, b1, W2, b2, W3, b3 = unpack(wq)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x)
    a, z, l = forward(x, wq)
    loss = np.mean(np.maximum(l, 0) - l * y + np.log1p(np.exp(-np.abs(l))))
    dl = (1.0 / (1.0 + np.exp(-l)) - y) / n
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = dl @ z
    g[OFF_B3] = dl.sum()
    dz = np.outer(dl, W3) * (z > 0)
    g[OFF_W2:OFF_B2] = (dz.T @ a).ravel()
    g[OFF_B2:OFF_W3] = dz.sum(0)
    da = (dz @ W2) * (a > 0)
    g[OFF_W1:OFF_B1] = (da.T @ x).ravel()
    g[OFF_B1:OFF_W2] = da.sum(0)
    return loss, g


def loss_only(x, y, wq):
    """The loss for already-rounded weights (finite-difference checks perturb these)."""
    _, _, l = forward(x, wq)
    y = np.asarray(y, np.float64)
    return np.mean(np.maximum(l, 0) - l * y + np.log1p(np.exp(-np.abs(l))))


def probabilities(x, w, mean, inv_std):
    xs = (np.asarray(x, np.float64) - mean) * inv_std
    _, _, l = forward(xs, rounded(w))
    return 1.0 / (1.0 + np.exp(-l))
