"""GPU parity of the row-group SpMM (plans created with PLAN_ROW_GROUPS):
DETERMINISTIC products equal the oracle bit for bit -- every row still adds
its entries in stored order -- for every group size the autotuner can pick,
ragged shapes (empty rows, long rows, a last group shorter than R), FP32 and
FP64 and several k; BACKEND_DEFAULT stays within
|c - c_ref| <= gamma_{n+2} (|alpha| sum|a b| + |c0|) of the long-double
oracle."""

import numpy as np
import pytest

import oracle
from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import (PLAN_HAS_ROW_GROUPS, PLAN_ROW_GROUPS, SPMM_AUTO, SPMM_STAGED,
                               Determinism, SparseBlasTranspose)
from asc_cpp_b200.sparse_cuda import AscError, CsrPlan, CudaSpmm, DenseMatrixView
from oracle import CSR, OP_NONE, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, host

pytestmark = pytest.mark.gpu


def shapes(rng, dt):
    yield "irregular", synthetic.random_csr(rng, 1003, 900, 40, dt, 0.15)
    lengths = rng.integers(0, 30, size=517)
    lengths[[0, 7, 200, 516]] = [700, 1, 0, 1500]
    ptr, idx = synthetic._unique_sorted_rows(rng, 2000, lengths)
    yield "long_rows", synthetic.Csr(517, 2000, ptr, idx,
                                     rng.standard_normal(int(ptr[-1])).astype(dt))
    yield "stencil", synthetic.stencil_27(12, seed=3, dtype=dt)


def spmm(ctx, plan, a, b, c0, alpha, k):
    c = dev(c0)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, alpha, a,
             DenseMatrixView(dev(b), a.columns, k, writable=False), DenseMatrixView(c, a.rows, k),
             plan=plan)
    return host(c)


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("k", [4, 8, 32, 128, 260])
def test_row_groups_bit_exact_every_group_size(cuda_lib, restatement, dt, k):
    rng = np.random.default_rng(k)
    ctx = context()
    for name, a_h in shapes(rng, dt):
        if k % (4 if dt == np.float32 else 2):
            continue
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        want = c0.copy()
        restatement.standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                                  -1.25, b, ROW_MAJOR, k, want, ROW_MAJOR, k, k)
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
        got = spmm(ctx, plan, a, b, c0, -1.25, k)
        assert bits_equal(got, want), (name, "plan defaults")
        for r in (2, 4, 8, 16, 32):  # every group size, chosen explicitly
            plan.set_spmm(r)
            assert plan.properties() & PLAN_HAS_ROW_GROUPS
            assert bits_equal(spmm(ctx, plan, a, b, c0, -1.25, k), want), (name, r)
        # the autotuner's candidates, then the one it keeps
        scratch = dev(c0)
        ms, rg = plan.spmm_autotune(0.5, DenseMatrixView(dev(b), a_h.cols, k, writable=False),
                                    DenseMatrixView(scratch, a_h.rows, k), reps=1)
        assert rg in (0, SPMM_STAGED, 2, 4, 8, 16, 32) and ms > 0
        assert bits_equal(spmm(ctx, plan, a, b, c0, -1.25, k), want), (name, rg)
        plan.close()
    ctx.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_row_groups_default_mode_within_bound(cuda_lib, restatement, dt):
    rng = np.random.default_rng(11)
    ctx = context(Determinism.kBackendDefault)
    k = 16
    for name, a_h in shapes(rng, dt):
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
        plan.set_spmm(8)
        got = spmm(ctx, plan, a, b, c0, 0.75, k)
        counts = np.diff(a_h.ptr)
        for j in range(k):
            bj = np.ascontiguousarray(b[:, j])
            exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                                 a_h.val, bj)
            ref = c0[:, j].astype(np.longdouble) + 0.75 * exact
            rep = oracle.error_report(got[:, j], ref, absval, counts, dt, 0.75,
                                      np.abs(c0[:, j].astype(np.float64)))
            assert rep["max_ratio_to_bound"] <= 1.0, (name, j, rep)
        plan.close()
    ctx.close()


def test_groups_only_when_chosen(cuda_lib):
    """Row groups run only when chosen (set_spmm or the autotuner); a plan
    starts on its default kernels, and SPMM_AUTO returns to them."""
    a_h = synthetic.stencil_27(16, seed=2, dtype=np.float32)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    assert not plan.properties() & PLAN_HAS_ROW_GROUPS
    plan.set_spmm(8)
    assert plan.properties() & PLAN_HAS_ROW_GROUPS
    b = np.random.default_rng(1).standard_normal((a_h.cols, 8)).astype(np.float32)
    c0 = np.zeros((a_h.rows, 8), np.float32)
    got = spmm(ctx, plan, a, b, c0, 1.0, 8)
    want = c0.copy()
    oracle.Restatement().standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                       a_h.val, 1.0, b, ROW_MAJOR, 8, want, ROW_MAJOR, 8, 8)
    assert bits_equal(got, want)
    plan.set_spmm(SPMM_AUTO)
    assert not plan.properties() & PLAN_HAS_ROW_GROUPS
    with pytest.raises(AscError):
        plan.set_spmm(3)
    plan.close()
    ctx.close()
