"""Seeded synthetic CSR workloads.

The reference publishes no matrices or datasets for this path, so every
workload is generated here from a seed.  Layout is the reference's canonical
CSR (include/asc/sparse/compressed.h:143-215,711-746): int64 ``ptr[rows+1]``
starting at 0, int64 column ``idx[nnz]`` sorted and unique within each row,
values ``val[nnz]``.

Workloads:

* :func:`laplacian_2d` - 5-point Laplacian on an ``m x m`` grid (diag 4,
  off-diagonals -1).  ``m = 316`` gives 99,856 rows and 498,016 nonzeros.
* :func:`power_law` - square matrix whose row lengths are lognormal with
  arithmetic mean ``mean`` and shape ``sigma`` (mu = ln(mean) - sigma^2/2),
  rounded and clipped to ``[1, max_len]``; columns uniform without
  replacement and sorted; values N(0,1).
* :func:`stencil_27` - 27-point stencil on an ``m^3`` grid, values N(0,1).
* :func:`block_sparse` - dense ``b x b`` blocks at a given block density.
* :func:`banded_batch` - many banded matrices with sparse off-band fill.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Csr:
    rows: int
    cols: int
    ptr: np.ndarray  # int64[rows+1]
    idx: np.ndarray  # int64[nnz]
    val: np.ndarray  # float32/float64[nnz]

    @property
    def nnz(self) -> int:
        return int(self.ptr[-1])

    def astype(self, dtype) -> "Csr":
        return Csr(self.rows, self.cols, self.ptr, self.idx,
                   self.val.astype(dtype))

    def bytes_spmv(self, elem: int, y_reads: bool = False) -> int:
        """Algorithmic bytes of one SpMV: nnz*(val+idx) + (n+1)*ptr + |x| + |y|."""
        b = self.nnz * (elem + 8) + (self.rows + 1) * 8
        b += self.cols * elem + self.rows * elem
        if y_reads:
            b += self.rows * elem
        return b


def laplacian_2d(m: int = 316, dtype=np.float64) -> Csr:
    n = m * m
    i, j = np.divmod(np.arange(n, dtype=np.int64), m)
    # columns of each row in increasing order: up, left, centre, right, down
    offs = np.array([-m, -1, 0, 1, m], dtype=np.int64)
    vals = np.array([-1.0, -1.0, 4.0, -1.0, -1.0])
    valid = np.stack([i > 0, j > 0, np.ones(n, bool), j < m - 1, i < m - 1],
                     axis=1)
    cols = np.arange(n, dtype=np.int64)[:, None] + offs[None, :]
    counts = valid.sum(axis=1)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    idx = cols[valid]
    val = np.broadcast_to(vals, (n, 5))[valid].astype(dtype)
    return Csr(n, n, ptr, idx, val)


def _unique_sorted_rows(rng: np.random.Generator, n_cols: int,
                        lengths: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per row, ``lengths[r]`` distinct uniform columns in [0, n_cols), sorted."""
    rows = lengths.size
    lengths = np.minimum(lengths, n_cols).astype(np.int64)
    total = int(lengths.sum())
    row_of = np.repeat(np.arange(rows, dtype=np.int64), lengths)
    cols = rng.integers(0, n_cols, size=total, dtype=np.int64)
    key = row_of * n_cols + cols
    key.sort()
    dup = np.zeros(total, dtype=bool)
    dup[1:] = key[1:] == key[:-1]
    if dup.any():
        # redraw the duplicates of each affected row (rare) until unique
        key = key[~dup]
        have = np.bincount(key // n_cols, minlength=rows)
        short = np.nonzero(have < lengths)[0]
        extra = []
        for r in short:
            base = key[np.searchsorted(key, r * n_cols):
                       np.searchsorted(key, (r + 1) * n_cols)] - r * n_cols
            need = int(lengths[r] - have[r])
            chosen = set(base.tolist())
            fresh = []
            while len(fresh) < need:
                c = int(rng.integers(0, n_cols))
                if c not in chosen:
                    chosen.add(c)
                    fresh.append(c)
            extra.append(r * n_cols + np.array(fresh, dtype=np.int64))
        key = np.sort(np.concatenate([key] + extra))
    ptr = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(lengths, out=ptr[1:])
    return ptr, key % n_cols


def power_law(n: int = 4_194_304, mean: float = 16.0, sigma: float = 1.5,
              max_len: int = 65_536, seed: int = 1, dtype=np.float64) -> Csr:
    rng = np.random.default_rng(seed)
    mu = np.log(mean) - sigma * sigma / 2.0
    lengths = np.rint(rng.lognormal(mu, sigma, size=n))
    lengths = np.clip(lengths, 1, max_len).astype(np.int64)
    ptr, idx = _unique_sorted_rows(rng, n, lengths)
    val = rng.standard_normal(int(ptr[-1])).astype(dtype)
    return Csr(n, n, ptr, idx, val)


def stencil_27(m: int = 128, seed: int = 2, dtype=np.float32) -> Csr:
    n = m ** 3
    rng = np.random.default_rng(seed)
    g = np.arange(n, dtype=np.int64)
    k, rem = np.divmod(g, m * m)
    i, j = np.divmod(rem, m)
    cols_list, valid_list = [], []
    for dk in (-1, 0, 1):
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                ok = ((k + dk >= 0) & (k + dk < m) & (i + di >= 0) &
                      (i + di < m) & (j + dj >= 0) & (j + dj < m))
                cols_list.append(g + dk * m * m + di * m + dj)
                valid_list.append(ok)
    cols = np.stack(cols_list, axis=1)  # already increasing per row
    valid = np.stack(valid_list, axis=1)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(valid.sum(axis=1), out=ptr[1:])
    idx = cols[valid]
    val = rng.standard_normal(idx.size).astype(dtype)
    return Csr(n, n, ptr, idx, val)


def block_sparse(rows: int = 65_536, block: int = 16, density: float = 0.02,
                 seed: int = 2, dtype=np.float32) -> Csr:
    """Square matrix made of dense ``block x block`` tiles; each block row
    holds round(density * block_cols) distinct block columns (sorted)."""
    rng = np.random.default_rng(seed)
    nb = rows // block
    per = max(1, int(round(density * nb)))
    lengths = np.full(nb, per, dtype=np.int64)
    bptr, bidx = _unique_sorted_rows(rng, nb, lengths)
    # expand: row r of block row R has entries bidx[k]*block + 0..block-1
    b_of_row = np.repeat(np.arange(nb, dtype=np.int64), block)
    row_len = per * block
    ptr = np.arange(rows + 1, dtype=np.int64) * row_len
    blocks_of_row = bidx.reshape(nb, per)[b_of_row]  # [rows, per]
    idx = (blocks_of_row[:, :, None] * block +
           np.arange(block, dtype=np.int64)[None, None, :]).reshape(-1)
    val = rng.standard_normal(idx.size).astype(dtype)
    return Csr(rows, rows, ptr, idx, val)


def banded(rng: np.random.Generator, n: int, half_band: int,
           fill: float = 0.01, dtype=np.float64) -> Csr:
    """Banded n x n matrix (|i-j| <= half_band) plus round(fill * band nnz)
    uniform off-band entries, deduplicated against the band."""
    r = np.arange(n, dtype=np.int64)
    lo = np.maximum(r - half_band, 0)
    hi = np.minimum(r + half_band, n - 1)
    band_len = hi - lo + 1
    band_nnz = int(band_len.sum())
    n_fill = int(round(fill * band_nnz))
    fr = rng.integers(0, n, size=n_fill, dtype=np.int64)
    fc = rng.integers(0, n, size=n_fill, dtype=np.int64)
    off = np.abs(fr - fc) > half_band
    fr, fc = fr[off], fc[off]
    band_rows = np.repeat(r, band_len)
    band_cols = (np.arange(band_nnz, dtype=np.int64) -
                 np.repeat(np.cumsum(band_len) - band_len, band_len) +
                 np.repeat(lo, band_len))
    key = np.unique(np.concatenate([band_rows * n + band_cols, fr * n + fc]))
    rows_of = key // n
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows_of, minlength=n), out=ptr[1:])
    idx = key % n
    val = rng.standard_normal(idx.size).astype(dtype)
    return Csr(n, n, ptr, idx, val)


def banded_batch(count: int = 4096, min_rows: int = 64, max_rows: int = 16_384,
                 max_half_band: int = 31, seed: int = 3,
                 dtype=np.float64) -> list[Csr]:
    rng = np.random.default_rng(seed)
    sizes = rng.integers(min_rows, max_rows + 1, size=count)
    bands = rng.integers(1, max_half_band + 1, size=count)
    return [banded(rng, int(n), int(b), dtype=dtype)
            for n, b in zip(sizes, bands)]


def uniform_vector(n: int, seed: int, dtype=np.float64,
                   rng: np.random.Generator | None = None) -> np.ndarray:
    rng = rng or np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=n).astype(dtype)


def random_csr(rng: np.random.Generator, rows: int, cols: int,
               max_len: int, dtype=np.float64, empty_frac: float = 0.0) -> Csr:
    """Small irregular CSR for parity tests (empty rows allowed)."""
    lengths = rng.integers(0, max_len + 1, size=rows)
    if empty_frac > 0:
        lengths[rng.random(rows) < empty_frac] = 0
    lengths = np.minimum(lengths, cols)
    ptr, idx = _unique_sorted_rows(rng, max(cols, 1), lengths)
    val = rng.standard_normal(int(ptr[-1])).astype(dtype)
    return Csr(rows, cols, ptr, idx, val)
