"""asc_sb_csr_spmv_no_alloc: the SpMV entry point for callers that cannot
allocate device memory or hand in a workspace (plugin hosts whose device
memory belongs to the host application's allocator, latency-critical loops
that must not take a cudaMalloc/cudaFree synchronisation).  Its partition
scratch is a static device array, so it takes no workspace; its results must
equal asc_sb_csr_spmv's.

This file is collected last on purpose: it touches process-wide state (the
shared static scratch), so a stop at the first failure has run everything
else already.  It also passes when run alone in a fresh process."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import Determinism, ErrorCode
from asc_cpp_b200.sparse_cuda import CudaCsrSpmv, CudaCsrSpmvWorkspaceSize

from gpu_util import bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu


def _no_alloc(ctx, alpha, a, x, beta, y):
    m, xd, yd = a.describe(), vec(x, writable=False).describe(), vec(y).describe()
    return ctx._lib.asc_sb_csr_spmv_no_alloc(ctx.handle, float(alpha), ctypes.byref(m),
                                             ctypes.byref(xd), float(beta), ctypes.byref(yd))


def _with_workspace(ctx, alpha, a, x, beta, y):
    xv, yv = vec(x, writable=False), vec(y)
    need = CudaCsrSpmvWorkspaceSize(ctx, a, xv, yv)
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    CudaCsrSpmv(ctx, alpha, a, xv, beta, yv, ws, need)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("determinism", [Determinism.kDeterministic,
                                         Determinism.kBackendDefault])
def test_no_alloc_matches_workspace_entry_point(cuda_lib, dt, determinism):
    """Two calls in a row (different matrices and scalars, so the second call
    overwrites the first call's scratch) equal the workspace entry point bit
    for bit, in both numerical modes."""
    rng = np.random.default_rng(31)
    ctx = context(determinism)
    cases = [synthetic.power_law(30000, seed=9, dtype=dt),
             synthetic.random_csr(rng, 5000, 3000, 300, dt, 0.2)]
    for a_h, (alpha, beta) in zip(cases, [(1.0, 0.0), (-0.5, 2.0)]):
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        x = dev(rng.uniform(-1, 1, a_h.cols).astype(dt))
        y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
        y_ref = dev(y0)
        _with_workspace(ctx, alpha, a, x, beta, y_ref)
        y = dev(y0)
        assert _no_alloc(ctx, alpha, a, x, beta, y) == 0, ctx._lib.asc_sb_context_last_error(ctx.handle)
        assert bits_equal(host(y), host(y_ref))
    assert ctx.device_status() == 0
    ctx.close()


def test_no_alloc_rejects_matrices_beyond_its_scratch(cuda_lib):
    """A matrix whose partition does not fit the static scratch is refused with
    kUnsupported before anything runs; y is untouched."""
    ctx = context()
    # needs ceil(2*rows/251) + 1 = 318,727 tile bounds (empty, so 16-byte
    # aligned, index and value arrays) > 262,144
    rows = 40_000_000
    ptr = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
    a = csr(2, 2, [0, 0, 0], np.zeros(0, np.int64), np.zeros(0))
    a.rows, a.columns, a.offsets = rows, 1, ptr
    x = dev(np.ones(1))
    y = torch.full((rows,), 7.0, dtype=torch.float64, device="cuda")
    rc = _no_alloc(ctx, 1.0, a, x, 0.0, y)
    assert rc == ErrorCode.kUnsupported
    assert b"static scratch" in ctx._lib.asc_sb_context_last_error(ctx.handle)
    assert bool((y == 7.0).all())
    ctx.close()
