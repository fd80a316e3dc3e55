"""GPU parity of the tensor-core SpMM for matrices made of dense 16 x 16
blocks (tcgen05, FP32 operands split into three TF32 products): plans detect
the block structure exactly, and results stay within the stated bound
|c - c_exact| <= (n + 64) 2^-22 |alpha| sum|a b| + 2^-23 |c0| against the
long-double oracle; DETERMINISTIC mode still runs the bit-exact kernel."""

import numpy as np
import pytest

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import PLAN_HAS_BLOCKS16, Determinism, SparseBlasTranspose
from asc_cpp_b200.sparse_cuda import CsrPlan, CudaSpmm, DenseMatrixView
from oracle import CSR, OP_NONE, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, host

pytestmark = pytest.mark.gpu


def block_matrix(rng, block_rows, block_cols, blocks_per_row):
    """Dense 16 x 16 blocks; blocks_per_row[i] distinct sorted block columns."""
    rows, cols = block_rows * 16, block_cols * 16
    ptr = [0]
    idx = []
    for br in range(block_rows):
        bcs = np.sort(rng.choice(block_cols, blocks_per_row[br], replace=False))
        row_cols = (bcs[:, None] * 16 + np.arange(16)[None, :]).reshape(-1)
        for _ in range(16):
            idx.append(row_cols)
            ptr.append(ptr[-1] + row_cols.size)
    idx = np.concatenate(idx).astype(np.int64) if idx else np.zeros(0, np.int64)
    val = rng.standard_normal(idx.size).astype(np.float32)
    return synthetic.Csr(rows, cols, np.array(ptr, np.int64), idx, val)


def check_bound(restatement, a_h, b, c0, out, alpha):
    counts = np.diff(a_h.ptr)
    for j in range(b.shape[1]):
        bj = np.ascontiguousarray(b[:, j])
        exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                             a_h.val, bj)
        ref = c0[:, j].astype(np.float64) + alpha * exact.astype(np.float64)
        bound = ((counts + 64) * 2.0 ** -22 * abs(alpha) * absval.astype(np.float64) +
                 2.0 ** -23 * np.abs(c0[:, j]) + np.finfo(np.float32).tiny)
        err = np.abs(out[:, j].astype(np.float64) - ref)
        assert np.all(err <= bound), (j, float(np.max(err / bound)))


@pytest.mark.parametrize("k", [1, 8, 32, 64, 100, 128, 200, 260])
def test_tensor_core_spmm_within_bound(cuda_lib, restatement, k):
    rng = np.random.default_rng(200 + k)
    a_h = block_matrix(rng, 48, 40, rng.integers(0, 9, 48))  # includes empty block rows
    b = rng.standard_normal((a_h.cols, k)).astype(np.float32)
    c0 = rng.standard_normal((a_h.rows, k)).astype(np.float32)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a)
    assert plan.properties() & PLAN_HAS_BLOCKS16
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, -0.75, a,
             DenseMatrixView(dev(b), a_h.cols, k, writable=False),
             DenseMatrixView(c, a_h.rows, k), plan=plan)
    check_bound(restatement, a_h, b, c0, host(c), -0.75)
    assert ctx.device_status(clear=True) == 0
    # DETERMINISTIC keeps the bit-exact stored-order kernel
    ctx.set_determinism(Determinism.kDeterministic)
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, -0.75, a,
             DenseMatrixView(dev(b), a_h.cols, k, writable=False),
             DenseMatrixView(c, a_h.rows, k), plan=plan)
    expect = c0.copy()
    restatement.standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                              -0.75, b, ROW_MAJOR, k, expect, ROW_MAJOR, k, k)
    assert bits_equal(host(c), expect)
    plan.close()
    ctx.close()


def test_block_sparse_config_shape_sample(cuda_lib, restatement):
    """The block-sparse generator's matrices (2% block density) are detected
    and multiplied within the bound (a 4096-row sample, k = 128)."""
    a_h = synthetic.block_sparse(rows=4096, block=16, density=0.02, seed=2)
    rng = np.random.default_rng(2)
    k = 128
    b = rng.standard_normal((a_h.cols, k)).astype(np.float32)
    c0 = np.zeros((a_h.rows, k), np.float32)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a)
    assert plan.properties() & PLAN_HAS_BLOCKS16
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, a,
             DenseMatrixView(dev(b), a_h.cols, k, writable=False),
             DenseMatrixView(c, a_h.rows, k), plan=plan)
    check_bound(restatement, a_h, b, c0, host(c), 1.0)
    plan.close()
    ctx.close()


def test_structure_detection_is_exact(cuda_lib):
    rng = np.random.default_rng(7)
    ctx = context(Determinism.kBackendDefault)
    good = block_matrix(rng, 10, 12, rng.integers(1, 5, 10))
    a = csr(good.rows, good.cols, good.ptr, good.idx, good.val)
    plan = CsrPlan(ctx, a)
    assert plan.properties() & PLAN_HAS_BLOCKS16
    plan.close()
    # drop the last entry of one row: no longer dense blocks
    ptr = good.ptr.copy()
    r = 37
    cut = ptr[r + 1] - 1
    idx = np.delete(good.idx, cut)
    val = np.delete(good.val, cut)
    ptr[r + 1:] -= 1
    bad = csr(good.rows, good.cols, ptr, idx, val)
    plan = CsrPlan(ctx, bad)
    assert not plan.properties() & PLAN_HAS_BLOCKS16
    plan.close()
    # shifted columns (blocks not aligned to 16)
    shifted = csr(good.rows, good.cols + 1, good.ptr, good.idx + 1, good.val)
    plan = CsrPlan(ctx, shifted)
    assert not plan.properties() & PLAN_HAS_BLOCKS16
    plan.close()
    # FP64 matrices and row counts not a multiple of 16 are never marked
    plan = CsrPlan(ctx, csr(good.rows, good.cols, good.ptr, good.idx, good.val.astype(np.float64)))
    assert not plan.properties() & PLAN_HAS_BLOCKS16
    plan.close()
    ctx.close()
