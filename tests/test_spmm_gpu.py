"""GPU parity of the SpMM entry point: the stored-order kernels are bit-exact
against the reference (golden cases) and the oracle; scatter (transposed)
products stay within the error bound."""

import numpy as np
import pytest

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import Determinism, ErrorCode, SparseBlasLayout, SparseBlasTranspose
from asc_cpp_b200.sparse_cuda import AscError, CudaSpmm, DenseMatrixView
from oracle import COL_MAJOR, CSR, OP_NONE, OP_TRANSPOSE, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, gamma, host

pytestmark = pytest.mark.gpu


def test_golden_spmm_cases(cuda_lib, random_cases):
    ctx = context()
    for case in range(int(random_cases["count"][0])):
        p = f"c{case}_"
        rows, cols = (int(v) for v in random_cases[p + "shape"])
        alpha = float(random_cases[p + "ab"][0])
        c0 = random_cases[p + "c0"]
        k = c0.size // rows
        a = csr(rows, cols, random_cases[p + "ptr"], random_cases[p + "idx"],
                random_cases[p + "val"])
        c = dev(c0)
        CudaSpmm(ctx, SparseBlasTranspose.kNone, alpha, a,
                 DenseMatrixView(dev(random_cases[p + "b"]), cols, k, writable=False),
                 DenseMatrixView(c, rows, k))
        assert bits_equal(host(c), random_cases[p + "spmm"]), case
    ctx.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("k", [1, 8, 32, 40, 128, 300])
def test_row_major_bit_exact(cuda_lib, restatement, dt, k):
    rng = np.random.default_rng(k)
    a_h = synthetic.random_csr(rng, 700, 500, 40, dt, 0.1)
    b = rng.uniform(-1, 1, (a_h.cols, k)).astype(dt)
    c0 = rng.uniform(-1, 1, (a_h.rows, k)).astype(dt)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, -0.5, a,
             DenseMatrixView(dev(b), a_h.cols, k, writable=False), DenseMatrixView(c, a_h.rows, k))
    expect = c0.copy()
    restatement.standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val, -0.5,
                              b, ROW_MAJOR, k, expect, ROW_MAJOR, k, k)
    assert bits_equal(host(c), expect)
    ctx.close()


def test_column_major_and_padded_ld_bit_exact(cuda_lib, restatement):
    rng = np.random.default_rng(4)
    a_h = synthetic.random_csr(rng, 300, 260, 25, np.float64, 0.1)
    k, ldb, ldc = 5, 270, 301
    b = rng.uniform(-1, 1, ldb * k)
    c0 = rng.uniform(-1, 1, ldc * k)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, 2.0, a,
             DenseMatrixView(dev(b), a_h.cols, k, SparseBlasLayout.kColumnMajor, ldb, False),
             DenseMatrixView(c, a_h.rows, k, SparseBlasLayout.kColumnMajor, ldc))
    expect = c0.copy()
    restatement.standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val, 2.0,
                              b, COL_MAJOR, ldb, expect, COL_MAJOR, ldc, k)
    out = host(c)
    assert bits_equal(out, expect)
    ctx.close()


def test_transposed_spmm_default_mode_within_bound(cuda_lib, restatement):
    rng = np.random.default_rng(12)
    a_h = synthetic.random_csr(rng, 400, 350, 30, np.float64, 0.1)
    k = 8
    b = rng.uniform(-1, 1, (a_h.rows, k))
    c0 = rng.uniform(-1, 1, (a_h.cols, k))
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kTranspose, 1.0, a,
             DenseMatrixView(dev(b), a_h.rows, k, writable=False), DenseMatrixView(c, a_h.cols, k))
    out = host(c)
    counts = restatement.output_counts(OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx)
    for j in range(k):
        bj = np.ascontiguousarray(b[:, j])
        exact, absval = restatement.extended(OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                             a_h.val, bj)
        ref = c0[:, j].astype(np.longdouble) + exact  # long double: exact to the bound
        bound = gamma(counts + 2, np.float64) * (absval.astype(np.float64) + np.abs(c0[:, j]))
        err = np.abs(out[:, j].astype(np.longdouble) - ref).astype(np.float64)
        assert np.all(err <= bound + 1e-300)
    ctx.close()


def test_spmm_shape_error(cuda_lib):
    ctx = context()
    a = csr(2, 2, [0, 1, 2], [0, 1], np.array([1.0, 2.0]))
    with pytest.raises(AscError) as e:
        CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, a,
                 DenseMatrixView(dev(np.ones(6)), 3, 2, writable=False),
                 DenseMatrixView(dev(np.ones(4)), 2, 2))
    assert e.value.code == ErrorCode.kShape
    ctx.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("k", [4, 8, 12, 32, 128, 200, 6])
def test_row_major_default_mode_within_bound(cuda_lib, restatement, dt, k):
    """BACKEND_DEFAULT row-major SpMM (contracted, alpha applied once per
    output) stays within gamma_{n+2}(|alpha| |A| |B| + |C0|) of the exact
    product; k not a multiple of the 16-byte chunk takes the scalar kernel."""
    rng = np.random.default_rng(100 + k)
    a_h = synthetic.random_csr(rng, 900, 600, 50, dt, 0.1)
    b = rng.uniform(-1, 1, (a_h.cols, k)).astype(dt)
    c0 = rng.uniform(-1, 1, (a_h.rows, k)).astype(dt)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, -1.5, a,
             DenseMatrixView(dev(b), a_h.cols, k, writable=False), DenseMatrixView(c, a_h.rows, k))
    out = host(c)
    counts = restatement.output_counts(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx)
    for j in range(k):
        bj = np.ascontiguousarray(b[:, j])
        exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                             a_h.val, bj)
        ref = c0[:, j].astype(np.longdouble) - 1.5 * exact  # long double
        bound = gamma(counts + 2, dt) * (1.5 * absval.astype(np.float64) +
                                         np.abs(c0[:, j].astype(np.float64)))
        err = np.abs(out[:, j].astype(np.longdouble) - ref).astype(np.float64)
        assert np.all(err <= bound + np.finfo(dt).tiny), j
    ctx.close()
