"""GPU parity of the device format conversions (CSR <-> CSC, coordinates ->
CSR / CSC) and of the deterministic transposed products that run on the
transposed structure of a plan.  All integer results must be identical to the
reference's conversions; deterministic transposed SpMV / SpMM must equal the
reference's serial order bit for bit."""

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import (PLAN_TRANSPOSE, Determinism, ErrorCode, FormatKind,
                               SparseBlasTranspose)
from asc_cpp_b200.sparse_cuda import (AscError, CsrPlan, CudaConvertCompressed,
                                      CudaConvertCoordinates, CudaSpmm, CudaSpmv,
                                      DenseMatrixView)
from oracle import CSC, CSR, OP_NONE, OP_TRANSPOSE, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu

CASES = ("ka", "r1", "r2", "r3", "r4")


def arrays(m):
    return host(m.offsets), host(m.indices), host(m.values)


@pytest.mark.parametrize("name", CASES)
def test_conversions_equal_reference_fixtures(cuda_lib, conversions, name):
    g = conversions
    r, c = (int(v) for v in g[f"{name}_shape"])
    ctx = context()
    a = csr(r, c, g[f"{name}_csr_ptr"], g[f"{name}_csr_idx"], g[f"{name}_csr_val"])
    t = CudaConvertCompressed(ctx, a)
    assert t.format == FormatKind.kCsc
    for k, arr in zip(("ptr", "idx", "val"), arrays(t)):
        assert bits_equal(arr, g[f"{name}_csc_{k}"]), k
    back = CudaConvertCompressed(ctx, t)
    assert back.format == FormatKind.kCsr
    for k, arr in zip(("ptr", "idx", "val"), arrays(back)):
        assert bits_equal(arr, g[f"{name}_csc_to_csr_{k}"]), k
    coo = dev(g[f"{name}_coo"].reshape(-1, 2))
    for fmt, kind in (("csr", FormatKind.kCsr), ("csc", FormatKind.kCsc)):
        m = CudaConvertCoordinates(ctx, r, c, coo, dev(g[f"{name}_csr_val"]), kind)
        for k, arr in zip(("ptr", "idx", "val"), arrays(m)):
            assert bits_equal(arr, g[f"{name}_coo_to_{fmt}_{k}"]), (fmt, k)
    ctx.close()


@pytest.mark.parametrize("rows,cols,max_len", [
    (5000, 300, 40),          # 1 radix pass (cols <= 256 after the first pass bits)
    (3000, 70000, 30),        # 3 passes
    (400, 20_000_000, 12),    # 4 passes, very sparse columns
    (1, 1, 1), (0, 10, 0), (10, 0, 0),
])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_csr_to_csc_matches_oracle(cuda_lib, restatement, rows, cols, max_len, dt):
    rng = np.random.default_rng(rows + cols)
    if rows and cols:
        a_h = synthetic.random_csr(rng, rows, cols, max_len, dt, 0.1)
        ptr, idx, val = a_h.ptr, a_h.idx, a_h.val
    else:
        ptr = np.zeros(rows + 1, np.int64)
        idx = np.zeros(0, np.int64)
        val = np.zeros(0, dt)
    ctx = context()
    t = CudaConvertCompressed(ctx, csr(rows, cols, ptr, idx, val))
    want = restatement.convert_compressed(1, rows, cols, ptr, idx, val.astype(np.float64))
    got = arrays(t)
    assert bits_equal(got[0], want[0]) and bits_equal(got[1], want[1])
    assert bits_equal(got[2], want[2].astype(dt))
    ctx.close()


def test_unsorted_coordinates_keep_storage_order(cuda_lib, restatement):
    """Out-of-order coordinates (with repeats) group by outer index and keep
    their storage order inside each group, as the reference's loop does."""
    rng = np.random.default_rng(31)
    nnz, rows, cols = 20000, 700, 90000
    coo = np.stack([rng.integers(0, rows, nnz), rng.integers(0, cols, nnz)], 1).astype(np.int64)
    val = rng.standard_normal(nnz)
    ctx = context()
    for to_csc, kind in ((0, FormatKind.kCsr), (1, FormatKind.kCsc)):
        m = CudaConvertCoordinates(ctx, rows, cols, dev(coo), dev(val), kind)
        want = restatement.convert_coordinates(to_csc, rows, cols, coo, val)
        for got, w in zip(arrays(m), want):
            assert bits_equal(got, w)
    ctx.close()


def test_round_trip_power_law_1m(cuda_lib):
    """CSR -> CSC -> CSR is the identity (a size-independent property)."""
    a_h = synthetic.power_law(1 << 20, seed=1, dtype=np.float64)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    back = CudaConvertCompressed(ctx, CudaConvertCompressed(ctx, a))
    torch.cuda.synchronize()
    assert torch.equal(back.offsets, a.offsets)
    assert torch.equal(back.indices, a.indices)
    assert torch.equal(back.values.view(torch.int64), a.values.view(torch.int64))
    ctx.close()


def test_conversion_failures(cuda_lib):
    ctx = context()
    a = csr(3, 4, [0, 2, 4, 5], [1, 3, 0, 2, 1], np.array([2.0, -1, 4, 5, 3]))
    lib = ctx._lib
    import ctypes
    d_src = a.describe()
    same = csr(3, 4, [0, 0, 0, 0, 0][:4], np.zeros(5, np.int64), np.zeros(5))
    d_same = same.describe()
    n = ctypes.c_size_t()
    ctx.check(lib.asc_sb_convert_workspace_size(ctx.handle, 3, 4, 5, int(FormatKind.kCsc),
                                                ctypes.byref(n)))
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    # same format in and out
    rc = lib.asc_sb_convert_compressed(ctx.handle, ctypes.byref(d_src), ctypes.byref(d_same),
                                       ws.data_ptr(), n.value)
    assert rc == ErrorCode.kInvalidArgument
    # shape mismatch
    other = csr(4, 4, np.zeros(5, np.int64), np.zeros(5, np.int64), np.zeros(5),
                FormatKind.kCsc)
    d_other = other.describe()
    rc = lib.asc_sb_convert_compressed(ctx.handle, ctypes.byref(d_src), ctypes.byref(d_other),
                                       ws.data_ptr(), n.value)
    assert rc == ErrorCode.kShape
    # workspace too small: nothing written
    dst = csr(3, 4, np.full(5, 77, np.int64), np.full(5, 77, np.int64), np.full(5, 7.0),
              FormatKind.kCsc)
    d_dst = dst.describe()
    rc = lib.asc_sb_convert_compressed(ctx.handle, ctypes.byref(d_src), ctypes.byref(d_dst),
                                       ws.data_ptr(), n.value - 256)
    assert rc == ErrorCode.kInvalidArgument
    assert (host(dst.offsets) == 77).all() and (host(dst.values) == 7.0).all()
    # destination overlapping the source
    d_alias = dst.describe()
    d_alias.values = a.values.data_ptr()
    rc = lib.asc_sb_convert_compressed(ctx.handle, ctypes.byref(d_src), ctypes.byref(d_alias),
                                       ws.data_ptr(), n.value)
    assert rc == ErrorCode.kInvalidArgument
    ctx.close()


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_deterministic_transposed_spmv_through_plan(cuda_lib, restatement, dt):
    rng = np.random.default_rng(41)
    a_h = synthetic.random_csr(rng, 3000, 2200, 60, dt, 0.1)
    x_h = rng.uniform(-1, 1, a_h.rows).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.cols).astype(dt)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    expect = y0.copy()
    restatement.standard_spmv(CSR, OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                              -0.75, x_h, expect)
    # without a plan: the transposed structure is rebuilt in the context's scratch
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, -0.75, a, vec(dev(x_h), writable=False), vec(y))
    assert bits_equal(host(y), expect)
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE)
    for op in (SparseBlasTranspose.kTranspose, SparseBlasTranspose.kConjugateTranspose):
        y = dev(y0)
        CudaSpmv(ctx, op, -0.75, a, vec(dev(x_h), writable=False), vec(y), plan=plan)
        assert bits_equal(host(y), expect)
    # op = none through the same plan is unchanged
    x2 = rng.uniform(-1, 1, a_h.cols).astype(dt)
    y2 = rng.uniform(-1, 1, a_h.rows).astype(dt)
    e2 = y2.copy()
    restatement.standard_spmv(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val, 1.25,
                              x2, e2)
    yd = dev(y2)
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 1.25, a, vec(dev(x2), writable=False), vec(yd),
             plan=plan)
    assert bits_equal(host(yd), e2)
    # new values: refresh, then the transposed product follows them
    a.values.mul_(2)
    plan.refresh_values()
    expect2 = y0.copy()
    restatement.standard_spmv(CSR, OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                              (a_h.val * 2).astype(dt), -0.75, x_h, expect2)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, -0.75, a, vec(dev(x_h), writable=False), vec(y),
             plan=plan)
    assert bits_equal(host(y), expect2)
    plan.close()
    ctx.close()


def test_deterministic_csc_none_through_plan(cuda_lib, restatement):
    rng = np.random.default_rng(42)
    a_h = synthetic.random_csr(rng, 900, 1300, 40, np.float64, 0.2)  # arrays: CSC of 1300x900
    x_h = rng.uniform(-1, 1, a_h.rows)
    y0 = rng.uniform(-1, 1, a_h.cols)
    ctx = context()
    c = csr(a_h.cols, a_h.rows, a_h.ptr, a_h.idx, a_h.val, FormatKind.kCsc)
    plan = CsrPlan(ctx, c, PLAN_TRANSPOSE)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 0.5, c, vec(dev(x_h), writable=False), vec(y),
             plan=plan)
    expect = y0.copy()
    restatement.standard_spmv(CSC, OP_NONE, a_h.cols, a_h.rows, a_h.ptr, a_h.idx, a_h.val, 0.5,
                              x_h, expect)
    assert bits_equal(host(y), expect)
    plan.close()
    ctx.close()


@pytest.mark.parametrize("k", [1, 8, 32])
def test_deterministic_transposed_spmm_through_plan(cuda_lib, restatement, k):
    rng = np.random.default_rng(43 + k)
    a_h = synthetic.random_csr(rng, 700, 500, 30, np.float64, 0.1)
    b = rng.uniform(-1, 1, (a_h.rows, k))
    c0 = rng.uniform(-1, 1, (a_h.cols, k))
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kTranspose, 1.5, a,
             DenseMatrixView(dev(b), a_h.rows, k, writable=False), DenseMatrixView(c, a_h.cols, k),
             plan=plan)
    expect = c0.copy()
    restatement.standard_spmm(CSR, OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                              1.5, b, ROW_MAJOR, k, expect, ROW_MAJOR, k, k)
    assert bits_equal(host(c), expect)
    plan.close()
    ctx.close()
