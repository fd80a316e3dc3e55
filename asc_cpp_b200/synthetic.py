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
* :func:`triangular` - diagonally dominant triangular matrix, near-diagonal
  plus long-range entries; :func:`triangle_of` - one triangle of a matrix.
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


def banded_batch_device(count: int = 4096, min_rows: int = 64, max_rows: int = 16_384,
                        max_half_band: int = 31, fill: float = 0.01, seed: int = 3,
                        dtype=None, device=None, align: int = 4):
    """The banded batch generated on the GPU (same family as banded_batch:
    square n x n, n ~ U{min_rows..max_rows}, half band ~ U{1..max_half_band},
    round(fill * band nnz) uniform off-band entries, duplicates removed,
    values N(0,1)), for full-size runs where host generation would be slow.

    Returns a dict of device tensors: ``ptr`` (all matrices' offsets, each
    starting at 0), ``idx`` and ``val`` (each matrix's entries start at a
    multiple of ``align`` elements), ``x`` and ``y`` (concatenated, x
    uniform[-1, 1]), and per-matrix int64 numpy arrays ``rows``, ``nnz``,
    ``ptr_base``, ``nz_base`` and ``row_base``.  Sizes and bands come from a
    numpy generator seeded with ``seed``; entries from a torch CUDA generator
    with the same seed."""
    import torch
    dtype = dtype or torch.float64
    device = device or torch.device("cuda", 0)
    rng = np.random.default_rng(seed)
    sizes = rng.integers(min_rows, max_rows + 1, size=count).astype(np.int64)
    bands = rng.integers(1, max_half_band + 1, size=count).astype(np.int64)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    row_base = np.zeros(count + 1, np.int64)
    np.cumsum(sizes, out=row_base[1:])
    total_rows = int(row_base[-1])
    shift = int(max_rows - 1).bit_length()
    sizes_d = torch.from_numpy(sizes).to(device)
    bands_d = torch.from_numpy(bands).to(device)
    row_base_d = torch.from_numpy(row_base).to(device)
    mat_of_row = torch.repeat_interleave(torch.arange(count, device=device), sizes_d)
    r = torch.arange(total_rows, device=device) - row_base_d[:-1][mat_of_row]
    n_of_row = sizes_d[mat_of_row]
    b_of_row = bands_d[mat_of_row]
    lo = torch.clamp(r - b_of_row, min=0)
    hi = torch.minimum(r + b_of_row, n_of_row - 1)
    band_len = hi - lo + 1
    del n_of_row, hi
    band_total = int(band_len.sum())
    # band keys: global row << shift | column, already sorted
    start = torch.cumsum(band_len, 0) - band_len
    grow = torch.repeat_interleave(torch.arange(total_rows, device=device), band_len)
    col = torch.arange(band_total, device=device) - start[grow] + lo[grow]
    keys = (grow << shift) | col
    del grow, col, start, lo
    band_nnz = torch.zeros(count, dtype=torch.int64, device=device)
    band_nnz.index_add_(0, mat_of_row, band_len)
    del band_len, r, b_of_row, mat_of_row
    n_fill = torch.round(band_nnz.double() * fill).long()
    fill_total = int(n_fill.sum())
    if fill_total:
        fm = torch.repeat_interleave(torch.arange(count, device=device), n_fill)
        fn = sizes_d[fm]
        fr = (torch.rand(fill_total, generator=gen, device=device, dtype=torch.float64) * fn).long()
        fc = (torch.rand(fill_total, generator=gen, device=device, dtype=torch.float64) * fn).long()
        fr = torch.minimum(fr, fn - 1)
        fc = torch.minimum(fc, fn - 1)
        off = (fr - fc).abs() > bands_d[fm]
        fkeys = ((row_base_d[:-1][fm] + fr) << shift) | fc
        fkeys = torch.unique(fkeys[off])
        keys = torch.sort(torch.cat([keys, fkeys])).values
        del fm, fn, fr, fc, off, fkeys
    grow = keys >> shift
    col = keys & ((1 << shift) - 1)
    del keys
    counts = torch.bincount(grow, minlength=total_rows)
    gptr = torch.zeros(total_rows + 1, dtype=torch.int64, device=device)
    torch.cumsum(counts, 0, out=gptr[1:])
    del counts, grow
    nnz_base_plain = gptr[row_base_d].cpu().numpy()
    nnz = np.diff(nnz_base_plain)
    # rebased offsets: matrix m's ptr at ptr_base[m] .. ptr_base[m] + n_m
    ptr_base = row_base[:-1] + np.arange(count, dtype=np.int64)
    pm = torch.repeat_interleave(torch.arange(count, device=device), sizes_d + 1)
    local = torch.arange(int(ptr_base[-1] + sizes[-1] + 1), device=device) - \
        torch.from_numpy(ptr_base).to(device)[pm]
    grow0 = row_base_d[:-1][pm]
    ptr = gptr[grow0 + local] - gptr[grow0]
    del pm, local, grow0
    # entries moved so that every matrix starts at a multiple of `align`
    padded = (nnz + align - 1) // align * align
    nz_base = np.zeros(count + 1, np.int64)
    np.cumsum(padded, out=nz_base[1:])
    total_padded = int(nz_base[-1])
    total_nnz = int(nnz.sum())
    mat_of_entry = torch.repeat_interleave(torch.arange(count, device=device),
                                           torch.from_numpy(nnz).to(device))
    dest = torch.arange(total_nnz, device=device) - \
        torch.from_numpy(nnz_base_plain[:-1]).to(device)[mat_of_entry] + \
        torch.from_numpy(nz_base[:-1]).to(device)[mat_of_entry]
    del mat_of_entry
    idx = torch.zeros(total_padded, dtype=torch.int64, device=device)
    idx[dest] = col
    del col
    val = torch.zeros(total_padded, dtype=dtype, device=device)
    val[dest] = torch.randn(total_nnz, generator=gen, device=device,
                            dtype=torch.float64).to(dtype)
    del dest, gptr
    x = (torch.rand(total_rows, generator=gen, device=device, dtype=torch.float64) * 2 - 1).to(dtype)
    y = torch.zeros(total_rows, dtype=dtype, device=device)
    torch.cuda.synchronize(device)
    return {"ptr": ptr, "idx": idx, "val": val, "x": x, "y": y, "rows": sizes, "nnz": nnz,
            "ptr_base": ptr_base, "nz_base": nz_base[:-1], "row_base": row_base[:-1]}


def _values(rng: np.random.Generator, count: int, dtype) -> np.ndarray:
    v = rng.uniform(-1.0, 1.0, size=count)
    if np.iscomplexobj(np.zeros(1, dtype)):
        v = v + 1j * rng.uniform(-1.0, 1.0, size=count)
    return v.astype(dtype)


def triangular(rng: np.random.Generator, n: int, lower: bool = True, near: int = 4,
               far: int = 2, span: int = 64, dtype=np.float64,
               diagonal: bool = True) -> Csr:
    """Square triangular CSR: per row up to ``near`` entries within ``span``
    of the diagonal and ``far`` anywhere in the strict triangle (duplicates
    merged), values uniform in [-1, 1] (both parts for complex), and -- with
    ``diagonal`` -- a diagonal of magnitude 1 + sum of the row's |entries| with
    a random sign (a random phase for complex), so that solves stay well
    conditioned."""
    r = np.arange(n, dtype=np.int64)
    off = rng.integers(1, span + 1, size=(n, near), dtype=np.int64)
    cols_near = r[:, None] - off if lower else r[:, None] + off
    u = rng.random((n, far))
    if lower:
        cols_far = np.floor(u * r[:, None]).astype(np.int64)
        ok_far = r[:, None] > 0
    else:
        cols_far = r[:, None] + 1 + np.floor(u * (n - 1 - r)[:, None]).astype(np.int64)
        ok_far = r[:, None] < n - 1
    cols = np.concatenate([cols_near, cols_far], axis=1)
    ok = np.concatenate([(cols_near >= 0) & (cols_near < n),
                         np.broadcast_to(ok_far, cols_far.shape)], axis=1)
    key = np.unique((r[:, None] * n + cols)[ok])
    rows_of = key // n
    off_val = _values(rng, key.size, dtype)
    if diagonal:
        mag = np.bincount(rows_of, weights=np.abs(off_val), minlength=n) + 1.0
        if np.iscomplexobj(np.zeros(1, dtype)):
            sign = np.exp(1j * rng.uniform(0.0, 2.0 * np.pi, size=n))
        else:
            sign = rng.choice(np.array([-1.0, 1.0]), size=n)
        key = np.concatenate([key, r * n + r])
        order = np.argsort(key, kind="stable")
        key = key[order]
        off_val = np.concatenate([off_val, (sign * mag).astype(dtype)])[order]
        rows_of = key // n
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows_of, minlength=n), out=ptr[1:])
    return Csr(n, n, ptr, key % n, off_val)


def triangle_of(m: Csr, lower: bool = True) -> Csr:
    """The lower (or upper) triangle of a square CSR matrix, diagonal included."""
    rows_of = np.repeat(np.arange(m.rows, dtype=np.int64), np.diff(m.ptr))
    keep = m.idx <= rows_of if lower else m.idx >= rows_of
    ptr = np.zeros(m.rows + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows_of[keep], minlength=m.rows), out=ptr[1:])
    return Csr(m.rows, m.cols, ptr, m.idx[keep], m.val[keep])
