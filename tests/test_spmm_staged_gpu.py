"""GPU parity of the TMA-staged SpMM (plans created with PLAN_ROW_GROUPS on
matrices whose groups of 16 rows share columns): DETERMINISTIC products equal
the oracle bit for bit -- every row still adds its entries in stored order --
for FP32 and FP64, k from 4 to 260, ragged shapes (a row count that is not a
multiple of 16, empty rows, a long row), padded leading dimensions of B and C
(one bulk copy per row of B instead of one per segment) and every stage width
and level (with these shapes the kernel runs on wide groups of 64 rows at
k <= 16 (FP32) or 8 (FP64), on wide groups of 32 rows at k = 32 (FP32) or 16
(FP64), and mostly on 16-row groups above, where the stages fit);
BACKEND_DEFAULT stays within |c - c_ref| <= gamma_{n+2}(|alpha| sum|a b| +
|c0|) of the long-double oracle; a plan whose stages do not fit shared memory
for the call's k falls back to the other kernels with the same results."""

import numpy as np
import pytest
import torch

import oracle
from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import (PLAN_HAS_STAGED_SPMM, PLAN_ROW_GROUPS, SPMM_STAGED, Determinism,
                               SparseBlasTranspose)
from asc_cpp_b200.sparse_cuda import CsrPlan, CudaSpmm, DenseMatrixView
from oracle import CSR, OP_NONE, ROW_MAJOR

from gpu_util import bits_equal, context, csr, dev, host

pytestmark = pytest.mark.gpu


def staged_shapes(rng, dt):
    """Matrices whose groups share columns (the plan keeps the staged path)."""
    yield "stencil", synthetic.stencil_27(13, seed=3, dtype=dt)  # 2197 rows: ragged last group
    yield "laplacian", synthetic.laplacian_2d(37, dtype=dt)
    band = synthetic.banded(rng, 3001, 9, fill=0.002, dtype=dt)
    yield "banded", band
    # a banded matrix with empty rows and one long dense row
    n = 1500
    lengths = np.zeros(n, np.int64)
    rows = []
    for r in range(n):
        if r % 97 == 5:
            rows.append(np.zeros(0, np.int64))
        elif r == 700:
            rows.append(np.arange(0, n, 2, dtype=np.int64))
        else:
            lo, hi = max(0, r - 4), min(n, r + 5)
            rows.append(np.arange(lo, hi, dtype=np.int64))
        lengths[r] = rows[-1].size
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lengths, out=ptr[1:])
    idx = np.concatenate(rows)
    yield "ragged", synthetic.Csr(n, n, ptr, idx, rng.standard_normal(idx.size).astype(dt))


def run(ctx, plan, a, b, c0, alpha, ldb=None, ldc=None):
    """C += alpha A B with B and C stored with leading dimensions ldb / ldc
    (padding columns of B hold NaN: never read; of C: must stay untouched)."""
    k = b.shape[1]
    ldb = ldb or k
    ldc = ldc or k
    bs = np.full((b.shape[0], ldb), np.nan, b.dtype)
    bs[:, :k] = b
    cs = np.full((c0.shape[0], ldc), 7.0, c0.dtype)
    cs[:, :k] = c0
    bd, cd = dev(bs), dev(cs)
    CudaSpmm(ctx, SparseBlasTranspose.kNone, alpha, a,
             DenseMatrixView(bd, a.columns, k, leading_dimension=ldb, writable=False),
             DenseMatrixView(cd, a.rows, k, leading_dimension=ldc), plan=plan)
    out = host(cd)
    assert (out[:, k:] == 7.0).all()  # padding untouched
    return np.ascontiguousarray(out[:, :k])


def reference(restatement, a_h, b, c0, alpha):
    k = b.shape[1]
    want = c0.copy()
    restatement.standard_spmm(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val, alpha,
                              np.ascontiguousarray(b), ROW_MAJOR, k, want, ROW_MAJOR, k, k)
    return want


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("k", [4, 8, 16, 32, 64, 128, 260])
def test_staged_bit_exact(cuda_lib, restatement, dt, k):
    if k % (4 if dt == np.float32 else 2):
        pytest.skip("k must fill whole 16-byte chunks")
    rng = np.random.default_rng(100 + k)
    ctx = context()
    for name, a_h in staged_shapes(rng, dt):
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
        assert plan.properties() & PLAN_HAS_STAGED_SPMM, name
        plan.set_spmm(SPMM_STAGED)  # at every k, not only the default range
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        want = reference(restatement, a_h, b, c0, -1.25)
        assert bits_equal(run(ctx, plan, a, b, c0, -1.25), want), name
        plan.close()
    assert ctx.device_status() == 0
    ctx.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_staged_padded_leading_dimensions(cuda_lib, restatement, dt):
    """ldb != k: every row of B is its own bulk copy; ldc != k."""
    rng = np.random.default_rng(7)
    ctx = context()
    k = 8
    step = 4 if dt == np.float32 else 2
    for name, a_h in staged_shapes(rng, dt):
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
        plan.set_spmm(SPMM_STAGED)
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        want = reference(restatement, a_h, b, c0, 0.5)
        got = run(ctx, plan, a, b, c0, 0.5, ldb=k + 3 * step, ldc=k + step)
        assert bits_equal(got, want), name
        plan.close()
    ctx.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_staged_default_mode_within_bound(cuda_lib, restatement, dt):
    rng = np.random.default_rng(12)
    ctx = context(Determinism.kBackendDefault)
    k = 16
    for name, a_h in staged_shapes(rng, dt):
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
        plan.set_spmm(SPMM_STAGED)
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        got = run(ctx, plan, a, b, c0, 0.75)
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


def test_staged_chosen_by_autotuner_and_kept(cuda_lib, restatement):
    """The SpMM autotuner times the staged kernel among its candidates; the
    plan keeps whatever it picks, and products stay bit-exact."""
    rng = np.random.default_rng(13)
    a_h = synthetic.stencil_27(20, seed=4, dtype=np.float32)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    k = 32
    b = rng.standard_normal((a_h.cols, k)).astype(np.float32)
    c0 = rng.standard_normal((a_h.rows, k)).astype(np.float32)
    scratch = dev(c0)
    ms, rg = plan.spmm_autotune(1.0, DenseMatrixView(dev(b), a_h.cols, k, writable=False),
                                DenseMatrixView(scratch, a_h.rows, k), reps=2)
    assert rg in (0, SPMM_STAGED, 2, 4, 8, 16, 32) and ms > 0
    assert bool(plan.properties() & PLAN_HAS_STAGED_SPMM) == (rg == SPMM_STAGED)
    want = reference(restatement, a_h, b, c0, 2.0)
    assert bits_equal(run(ctx, plan, a, b, c0, 2.0), want)
    plan.close()
    ctx.close()


def test_stages_beyond_shared_memory_fall_back(cuda_lib, restatement):
    """Groups of 16 rows with 2000 distinct columns and 24,000 entries each:
    two stages need far more than a CTA's shared memory at any k, so the
    plan keeps the staged path (the groups share columns) but every product
    runs another kernel -- same bits."""
    rng = np.random.default_rng(14)
    n, cols = 64, 40_000
    rows = []
    for g in range(n // 16):
        base = rng.choice(cols, size=2000, replace=False)
        for _ in range(16):
            rows.append(np.sort(rng.choice(base, size=1500, replace=False)))
    lengths = np.array([r.size for r in rows])
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lengths, out=ptr[1:])
    idx = np.concatenate(rows).astype(np.int64)
    a_h = synthetic.Csr(n, cols, ptr, idx, rng.standard_normal(idx.size).astype(np.float32))
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    assert plan.properties() & PLAN_HAS_STAGED_SPMM
    plan.set_spmm(SPMM_STAGED)
    assert plan.spmm_stage_rows(4) == 0 and plan.spmm_stage_rows(128) == 0
    for k in (4, 128):
        b = rng.standard_normal((cols, k)).astype(np.float32)
        c0 = rng.standard_normal((n, k)).astype(np.float32)
        want = reference(restatement, a_h, b, c0, 1.0)
        assert bits_equal(run(ctx, plan, a, b, c0, 1.0), want), k
    plan.close()
    ctx.close()


def test_staged_bounded_wait_status_clean(cuda_lib):
    """Normal runs leave the context's status word clear (no stage wait gave
    up)."""
    a_h = synthetic.stencil_27(10, seed=5, dtype=np.float32)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    b = torch.ones((a_h.cols, 32), dtype=torch.float32, device="cuda")
    c = torch.zeros((a_h.rows, 32), dtype=torch.float32, device="cuda")
    for _ in range(3):
        CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, a, DenseMatrixView(b, a_h.cols, 32, writable=False),
                 DenseMatrixView(c, a_h.rows, 32), plan=plan)
    torch.cuda.synchronize()
    assert ctx.device_status() == 0
    plan.close()
    ctx.close()


# level (rows per group) the staged kernel runs on for a 27-point 40^3 stencil
# per k: of the levels whose two stages fit a CTA's shared memory (B200: 227
# KB), the one with the most CTAs per SM (228 KB per SM), the widest among
# equals (stage sizes from the groups' slot and entry counts)
LEVELS_40 = {np.float32: {4: 64, 16: 64, 32: 32, 128: 16},
             np.float64: {4: 64, 16: 32, 32: 16, 64: 16}}


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_stage_levels_bit_exact(cuda_lib, restatement, dt):
    """The staged kernel runs on wide groups of 64 or 32 rows (the columns
    their 16-row groups share merged into one slot: fewer, longer copies of
    B) or on the 16-row groups, by k; every level bit-exact."""
    rng = np.random.default_rng(21)
    ctx = context()
    a_h = synthetic.stencil_27(40, seed=6, dtype=dt)  # 64 000 rows
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    plan.set_spmm(SPMM_STAGED)
    for k, rows in LEVELS_40[dt].items():
        assert plan.spmm_stage_rows(k) == rows, k
        b = rng.standard_normal((a_h.cols, k)).astype(dt)
        c0 = rng.standard_normal((a_h.rows, k)).astype(dt)
        want = reference(restatement, a_h, b, c0, 0.625)
        assert bits_equal(run(ctx, plan, a, b, c0, 0.625), want), k
    assert ctx.device_status() == 0
    plan.close()
    ctx.close()


def test_stage_rows_zero_where_staging_does_not_apply(cuda_lib):
    ctx = context()
    a_h = synthetic.stencil_27(12, seed=7, dtype=np.float32)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plain = CsrPlan(ctx, a, 0)
    assert plain.spmm_stage_rows(32) == 0  # no staged tables
    plain.close()
    plan = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    assert plan.spmm_stage_rows(6) == 0    # rows of B not whole 16-byte chunks
    assert plan.spmm_stage_rows(1024) == 0  # more than 128 chunks per row
    assert plan.spmm_stage_rows(32) == 32
    plan.close()
    ctx.close()
