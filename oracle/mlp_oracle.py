"""CPU oracle of the variant selector -- test infrastructure only.

A float64 numpy restatement of the selector's math, used by ``tests/`` as the
checker of the CUDA kernels (the reference has no counterpart: the selector is
new, so this restatement follows the library's own stated definitions):

* ``features`` -- the twelve matrix features, from the definitions stated in
  the library header (log2 sizes, row-length statistics, distance to the
  diagonal, diagonal fraction, 8-column block runs, empty rows, precision);
* ``forward`` / ``backward`` -- the MLP 12 -> 64 -> 64 -> V with ReLU and the
  mean-squared-error loss sum_s sum_v (y - t)^2 / (batch * V), with its exact
  gradient (checked against central finite differences in the CPU tests);
* ``adam`` -- one Adam step with bias correction.
"""

from __future__ import annotations

import numpy as np

FEATURES = 12
HIDDEN = 64


def param_count(v: int) -> int:
    return HIDDEN * FEATURES + HIDDEN + HIDDEN * HIDDEN + HIDDEN + v * HIDDEN + v


def split(p: np.ndarray, v: int):
    o = 0
    out = []
    for shape in ((HIDDEN, FEATURES), (HIDDEN,), (HIDDEN, HIDDEN), (HIDDEN,), (v, HIDDEN), (v,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def features(rows, cols, ptr, idx, element_bytes) -> np.ndarray:
    ptr = np.asarray(ptr, np.int64)
    idx = np.asarray(idx, np.int64)
    nnz = int(ptr[-1]) if len(ptr) else 0
    n = max(rows, 1)
    c = max(cols, 1)
    lengths = np.diff(ptr).astype(np.float64)
    row_of = np.repeat(np.arange(rows, dtype=np.int64), np.diff(ptr))
    dist = np.abs(idx - row_of)
    first = np.zeros(nnz, bool)
    first[ptr[:-1][np.diff(ptr) > 0]] = True
    prev_block = np.concatenate([[-1], idx[:-1] >> 3]) if nnz else np.zeros(0, np.int64)
    starts = first | ((idx >> 3) != prev_block)
    segs = int(starts.sum())
    mean = nnz / n
    var = float((lengths ** 2).sum()) / n - mean * mean
    cv = np.sqrt(max(var, 0.0)) / mean if mean > 0 else 0.0
    mn = min(rows, cols)
    f = np.array([
        np.log2(1.0 + rows), np.log2(1.0 + cols), np.log2(1.0 + nnz), np.log2(1.0 + mean),
        np.log2(1.0 + (lengths.max() if rows else 0.0)), np.log2(1.0 + cv),
        (dist.max() if nnz else 0) / c,
        (dist.sum() / nnz / c) if nnz else 0.0,
        (float((idx == row_of).sum()) / mn) if mn > 0 else 0.0,
        (nnz / (8.0 * segs)) if segs else 0.0,
        float((lengths == 0).sum()) / n,
        1.0 if element_bytes >= 8 else 0.0,
    ])
    return f


def forward(p: np.ndarray, x: np.ndarray, v: int):
    w1, b1, w2, b2, w3, b3 = split(np.asarray(p, np.float64), v)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    y = h2 @ w3.T + b3
    return h1, h2, y


def loss(p, x, t, v) -> float:
    y = forward(p, x, v)[2]
    return float(((y - t) ** 2).sum() / (x.shape[0] * v))


def backward(p: np.ndarray, x: np.ndarray, t: np.ndarray, v: int) -> np.ndarray:
    w1, b1, w2, b2, w3, b3 = split(np.asarray(p, np.float64), v)
    x = np.asarray(x, np.float64)
    h1, h2, y = forward(p, x, v)
    dy = 2.0 * (y - t) / (x.shape[0] * v)
    gw3 = dy.T @ h2
    gb3 = dy.sum(0)
    dh2 = (dy @ w3) * (h2 > 0)
    gw2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    gw1 = dh1.T @ x
    gb1 = dh1.sum(0)
    return np.concatenate([g.reshape(-1) for g in (gw1, gb1, gw2, gb2, gw3, gb3)])


def adam(p, g, m, s, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    s = b2 * s + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(s / (1 - b2 ** step)) + eps)
    return p, m, s
