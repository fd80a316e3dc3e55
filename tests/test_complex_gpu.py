"""GPU parity of the complex (C, Z) standard SpMV / SpMM paths against the
reference's complex products (fixtures from the reference itself) and the
oracle.  DETERMINISTIC results must be bit-identical; BACKEND_DEFAULT ones
must stay within a componentwise bound of the exact product."""

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import PLAN_TRANSPOSE, Determinism, ErrorCode, FormatKind, SparseBlasTranspose
from asc_cpp_b200.sparse_cuda import AscError, CsrPlan, CudaSpmm, CudaSpmv, DenseMatrixView
from oracle import COL_MAJOR, CSC, CSR, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu

TAGS = [("z", np.complex128), ("c", np.complex64)]
OPS = [SparseBlasTranspose.kNone, SparseBlasTranspose.kTranspose,
       SparseBlasTranspose.kConjugateTranspose]


@pytest.mark.parametrize("tag,dt", TAGS)
def test_complex_known_answers(cuda_lib, complex_cases, tag, dt):
    """standard_blas_test.cc:177-345 on the complex 2 x 2 matrix."""
    g = complex_cases
    ctx = context()
    val = np.array([2 + 1j, 1 - 1j, 3 + 0.5j], dt)
    a = csr(2, 2, [0, 1, 3], [0, 0, 1], val)
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE)
    x = dev(np.array([1 + 2j, -1 + 1j], dt))
    y = dev(np.zeros(2, dt))
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 1.0, a, vec(x, writable=False), vec(y))
    assert bits_equal(host(y), g[f"ka_spmv_csr_none_{tag}"])
    y = dev(np.zeros(2, dt))
    CudaSpmv(ctx, SparseBlasTranspose.kConjugateTranspose, 1.0, a, vec(x, writable=False),
             vec(y), plan=plan)
    assert bits_equal(host(y), g[f"ka_spmv_csr_conjt_{tag}"])
    c_arr = csr(2, 2, [0, 2, 3], [0, 1, 1], val, FormatKind.kCsc)
    cplan = CsrPlan(ctx, c_arr, PLAN_TRANSPOSE)
    y = dev(np.zeros(2, dt))
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 1.0, c_arr, vec(x, writable=False), vec(y),
             plan=cplan)
    assert bits_equal(host(y), g[f"ka_spmv_csc_none_{tag}"])
    c = dev(np.zeros(4, dt))
    CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, a,
             DenseMatrixView(dev(np.array([1, 2, 3, 4], dt)), 2, 2, writable=False),
             DenseMatrixView(c, 2, 2))
    assert bits_equal(host(c), g[f"ka_spmm_row_{tag}"])
    # CSC with the conjugate transpose reads the stored arrays as rows
    from asc_cpp_b200._abi import SparseBlasLayout
    c = dev(np.zeros(4, dt))
    CudaSpmm(ctx, SparseBlasTranspose.kConjugateTranspose, 1.0, c_arr,
             DenseMatrixView(dev(np.array([1, 3, 2, 4], dt)), 2, 2,
                             layout=SparseBlasLayout.kColumnMajor, writable=False),
             DenseMatrixView(c, 2, 2, layout=SparseBlasLayout.kColumnMajor))
    assert bits_equal(host(c), g[f"ka_spmm_csc_col_conjt_{tag}"])
    # alpha = 0 with a NaN matrix leaves y alone
    nan = csr(2, 2, [0, 1, 3], [0, 0, 1], np.full(3, np.nan + 1j * np.nan, dt))
    y = dev(np.array([7, 9], dt))
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 0.0, nan, vec(x, writable=False), vec(y))
    assert bits_equal(host(y), np.array([7, 9], dt))
    plan.close()
    cplan.close()
    ctx.close()


@pytest.mark.parametrize("tag,dt", TAGS)
def test_complex_random_deterministic_equals_reference(cuda_lib, complex_cases, tag, dt):
    g = complex_cases
    rows, cols = (int(v) for v in g[f"rand_shape_{tag}"])
    ctx = context()
    a = csr(rows, cols, g[f"rand_ptr_{tag}"], g[f"rand_idx_{tag}"], g[f"rand_val_{tag}"])
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE)
    alpha = 0.75 - 1.25j
    for op in OPS:
        o = int(op)
        y = dev(g[f"rand_y0_op{o}_{tag}"])
        CudaSpmv(ctx, op, alpha, a, vec(dev(g[f"rand_x_op{o}_{tag}"]), writable=False), vec(y),
                 plan=plan)
        assert bits_equal(host(y), g[f"rand_y_op{o}_{tag}"]), op
        b = g[f"rand_b_op{o}_{tag}"]
        c = dev(g[f"rand_c0_op{o}_{tag}"])
        CudaSpmm(ctx, op, alpha, a, DenseMatrixView(dev(b), b.shape[0], 5, writable=False),
                 DenseMatrixView(c, c.shape[0], 5), plan=plan)
        assert bits_equal(host(c), g[f"rand_c_op{o}_{tag}"]), op
    # without a plan the transposed structure is built in the context's scratch:
    # the same bits
    y = dev(g[f"rand_y0_op1_{tag}"])
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, alpha, a,
             vec(dev(g[f"rand_x_op1_{tag}"]), writable=False), vec(y))
    assert bits_equal(host(y), g[f"rand_y_op1_{tag}"])
    b = g["rand_b_op1_" + tag]
    c = dev(g[f"rand_c0_op1_{tag}"])
    CudaSpmm(ctx, SparseBlasTranspose.kTranspose, alpha, a,
             DenseMatrixView(dev(b), b.shape[0], 5, writable=False),
             DenseMatrixView(c, c.shape[0], 5))
    assert bits_equal(host(c), g[f"rand_c_op1_{tag}"])
    plan.close()
    ctx.close()


def _bound_check(got, ref_exact, absval, n, dt):
    u = np.finfo(np.float32 if dt == np.complex64 else np.float64).eps / 2
    g = (n + 4) * u / (1 - (n + 4) * u)
    err = np.abs(got.astype(np.complex128) - ref_exact)
    assert np.all(err <= g * absval * 2 + 1e-300)


@pytest.mark.parametrize("tag,dt", TAGS)
def test_complex_default_mode_within_bound(cuda_lib, restatement, tag, dt):
    """BACKEND_DEFAULT: rows in any order, transposed products by scatter."""
    rng = np.random.default_rng(61)
    a_h = synthetic.random_csr(rng, 1500, 1100, 70, np.float64, 0.1)
    val = (rng.standard_normal(a_h.nnz) + 1j * rng.standard_normal(a_h.nnz)).astype(dt)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, val)
    alpha = -0.5 + 2j
    for op in OPS:
        nx = a_h.cols if op == SparseBlasTranspose.kNone else a_h.rows
        ny = a_h.rows if op == SparseBlasTranspose.kNone else a_h.cols
        x = (rng.uniform(-1, 1, nx) + 1j * rng.uniform(-1, 1, nx)).astype(dt)
        y0 = (rng.uniform(-1, 1, ny) + 1j * rng.uniform(-1, 1, ny)).astype(dt)
        y = dev(y0)
        CudaSpmv(ctx, op, alpha, a, vec(dev(x), writable=False), vec(y))
        # exact reference in complex128 from the oracle's order on widened data
        ref = y0.astype(np.complex128).copy()
        restatement.standard_spmv(CSR, int(op), a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                  val.astype(np.complex128), alpha, x.astype(np.complex128), ref)
        absv = np.abs(y0).astype(np.complex128)
        restatement.standard_spmv(CSR, int(op), a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                  np.abs(val).astype(np.complex128), abs(alpha),
                                  np.abs(x).astype(np.complex128), absv)
        counts = restatement.output_counts(int(op), a_h.rows, a_h.cols, a_h.ptr, a_h.idx)
        _bound_check(host(y), ref, absv.real, counts, dt)
    ctx.close()
