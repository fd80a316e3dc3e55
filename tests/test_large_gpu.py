"""Maximum sizes: a CSR matrix with more than 2^31 stored entries (int64
positions past the 32-bit range), built on the device, multiplied in both
numerical modes, and checked row by row against a host formula on sampled
rows, including the rows around position 2^31.

Values and x are small dyadic numbers (v = k/256 with |k| <= 512, x = m/1024
with |m| <= 1024), so every product and every partial sum of a row is exact
in FP64: the expected y does not depend on summation order, and any
indexing error shows as a wrong value."""

import numpy as np
import pytest
import torch

from asc_cpp_b200._abi import Determinism
from asc_cpp_b200.sparse_cuda import (CudaCsrArray, CudaCsrSpmv, CudaCsrSpmvWorkspaceSize,
                                      CudaStridedVectorView, SparseCudaContext)

pytestmark = pytest.mark.gpu

ROWS = (1 << 25) + (1 << 16)  # 33,619,968 rows
PER_ROW = 64                   # nnz = 2,151,677,952 > 2^31
CHUNK = 1 << 27


def _value(p):
    return ((p * 2654435761) % 1024 - 512) / 256.0


def _x(c):
    return ((c * 40503) % 2048 - 1024) / 1024.0


def _expected(r):
    base = min(r, ROWS - PER_ROW)
    s = 0.0
    for j in range(PER_ROW):
        s += _value(PER_ROW * r + j) * _x(base + j)
    return s


@pytest.fixture(scope="module")
def big_matrix():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    free, _ = torch.cuda.mem_get_info(0)
    if free < 60 * (1 << 30):
        pytest.skip("needs about 45 GB of free device memory")
    dev = torch.device("cuda", 0)
    nnz = ROWS * PER_ROW
    ptr = torch.arange(ROWS + 1, dtype=torch.int64, device=dev) * PER_ROW
    idx = torch.empty(nnz, dtype=torch.int64, device=dev)
    val = torch.empty(nnz, dtype=torch.float64, device=dev)
    j = torch.arange(PER_ROW, dtype=torch.int64, device=dev)
    rows_per_chunk = CHUNK // PER_ROW
    for r0 in range(0, ROWS, rows_per_chunk):
        r1 = min(ROWS, r0 + rows_per_chunk)
        r = torch.arange(r0, r1, dtype=torch.int64, device=dev)
        base = torch.clamp(r, max=ROWS - PER_ROW)
        idx[r0 * PER_ROW:r1 * PER_ROW] = (base[:, None] + j[None, :]).reshape(-1)
        p = torch.arange(r0 * PER_ROW, r1 * PER_ROW, dtype=torch.int64, device=dev)
        val[r0 * PER_ROW:r1 * PER_ROW] = ((p * 2654435761) % 1024 - 512).to(torch.float64) / 256.0
        del r, base, p
    c = torch.arange(ROWS, dtype=torch.int64, device=dev)
    x = ((c * 40503) % 2048 - 1024).to(torch.float64) / 1024.0
    del c
    torch.cuda.synchronize()
    yield CudaCsrArray(ROWS, ROWS, ptr, idx, val), x
    del ptr, idx, val, x
    torch.cuda.empty_cache()


def _sample_rows():
    boundary = (1 << 31) // PER_ROW  # the row holding position 2^31
    rng = np.random.default_rng(7)
    rows = set(range(0, 200)) | set(range(ROWS - 200, ROWS))
    rows |= set(range(boundary - 100, boundary + 100))
    rows |= set(int(v) for v in rng.integers(0, ROWS, 2000))
    return np.array(sorted(rows), dtype=np.int64)


@pytest.mark.parametrize("det", [Determinism.kDeterministic, Determinism.kBackendDefault])
def test_spmv_beyond_int32_positions(cuda_lib, big_matrix, det):
    a, x = big_matrix
    assert a.nnz > (1 << 31)
    stream = torch.cuda.default_stream(0)
    ctx = SparseCudaContext.Create(0, stream=stream, determinism=det)
    y = torch.full((ROWS,), float("nan"), dtype=torch.float64, device=x.device)
    xv = CudaStridedVectorView(x, ROWS, writable=False)
    yv = CudaStridedVectorView(y, ROWS)
    ws_bytes = CudaCsrSpmvWorkspaceSize(ctx, a, xv, yv)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=x.device)
    CudaCsrSpmv(ctx, 1.0, a, xv, 0.0, yv, ws, ws_bytes)
    torch.cuda.synchronize()
    rows = _sample_rows()
    got = y[torch.from_numpy(rows).to(x.device)].cpu().numpy()
    want = np.array([_expected(int(r)) for r in rows])
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, [(int(rows[i]), got[i], want[i]) for i in bad[:5]]
    assert not torch.isnan(y).any()
    ctx.close()
