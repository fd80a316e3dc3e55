"""GPU tests of the ROW_SPLIT SpMV variant (BACKEND_DEFAULT): rows of 20,000
to 65,536 entries, whose tails past their tile are split into 256-entry
chunks over other warps, stay within
|y - y_ref| <= gamma_{n+2}(|alpha| sum|a x| + |beta y0|) of the long-double
oracle, repeat bit for bit run to run (partials are combined in a fixed
order), and agree across the workspace path, plans, the standard form and
every split threshold."""

import numpy as np
import pytest

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import Determinism, ErrorCode, SparseBlasTranspose, Variant
from asc_cpp_b200.sparse_cuda import AscError, CsrPlan, CudaCsrSpmv, CudaCsrSpmvWorkspaceSize, CudaSpmv
from oracle import OP_NONE

from gpu_util import assert_within_bound, bits_equal, context, csr, dev, host, vec

import torch

pytestmark = pytest.mark.gpu


def long_row_matrix(rng, dt, rows=3000, cols=1_000_000):
    """Mostly short rows (0..40 entries) with long rows of 20,000..65,536
    entries at scattered positions, including the first and last row and two
    adjacent long rows."""
    lengths = rng.integers(0, 41, size=rows)
    for r in (0, 1, 2, 17, 500, 501, rows * 2 // 3, rows - 1):
        lengths[r] = int(rng.integers(20_000, 65_537))
    lengths[2] = 65_536
    ptr, idx = synthetic._unique_sorted_rows(rng, cols, lengths)
    val = rng.standard_normal(int(ptr[-1])).astype(dt)
    return synthetic.Csr(rows, cols, ptr, idx, val)


def compat(ctx, a, alpha, x, beta, y):
    xv, yv = vec(x, writable=False), vec(y)
    need = CudaCsrSpmvWorkspaceSize(ctx, a, xv, yv)
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    CudaCsrSpmv(ctx, alpha, a, xv, beta, yv, ws, need)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["f64", "f32"])
def test_row_split_long_rows_within_bound_and_repeatable(cuda_lib, restatement, dt):
    rng = np.random.default_rng(77)
    a_h = long_row_matrix(rng, dt)
    x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
    alpha, beta = -1.5, 0.25
    exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                                         x_h)
    counts = np.diff(a_h.ptr)
    ref = alpha * exact + beta * y0.astype(np.longdouble)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    x = dev(x_h)
    results = {}
    for rounds in (0, 1, 2, 8, 32):
        ctx.set_variant(Variant.kRowSplit, rounds)
        for attempt in range(2):
            y = dev(y0)
            compat(ctx, a, alpha, x, beta, y)
            out = host(y)
            assert_within_bound(out, exact, absval, counts, dt, alpha,
                                np.abs(beta * y0.astype(np.float64)), ref)
            if attempt:
                assert bits_equal(out, results[rounds]), rounds  # run to run
            results[rounds] = out
        # the same threshold through a plan gives the same bits
        plan = CsrPlan(ctx, a)
        y = dev(y0)
        plan.csr_spmv(alpha, vec(x, writable=False), beta, vec(y))
        assert bits_equal(host(y), results[rounds]), ("plan", rounds)
        plan.close()
    assert ctx.device_status() == 0
    ctx.close()


def test_row_split_standard_form_through_plan(cuda_lib, restatement):
    """y += alpha*A*x with a plan (split block from the plan), and without a
    plan (no memory for the chunk table: rows run inline) -- both within the
    bound."""
    rng = np.random.default_rng(78)
    a_h = long_row_matrix(rng, np.float64, rows=1500)
    x_h = rng.uniform(-1, 1, a_h.cols)
    y0 = rng.uniform(-1, 1, a_h.rows)
    alpha = 0.75
    exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                                         x_h)
    counts = np.diff(a_h.ptr)
    ref = y0.astype(np.longdouble) + alpha * exact
    ctx = context(Determinism.kBackendDefault)
    ctx.set_variant(Variant.kRowSplit, 1)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a)
    for p in (plan, None):
        y = dev(y0)
        CudaSpmv(ctx, SparseBlasTranspose.kNone, alpha, a, vec(dev(x_h), writable=False), vec(y),
                 plan=p)
        assert_within_bound(host(y), exact, absval, counts, np.float64, alpha, np.abs(y0), ref)
    plan.close()
    ctx.close()


def test_row_split_short_rows_and_empty(cuda_lib, restatement):
    """Without long rows nothing is split and results equal WARP_TILES bit for
    bit."""
    rng = np.random.default_rng(79)
    a_h = synthetic.random_csr(rng, 20000, 9000, 50, np.float64, 0.2)
    x_h = rng.uniform(-1, 1, a_h.cols)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    outs = []
    for variant in (Variant.kWarpTiles, Variant.kRowSplit):
        ctx.set_variant(variant, 0)
        y = dev(np.zeros(a_h.rows))
        compat(ctx, a, 1.0, dev(x_h), 0.0, y)
        outs.append(host(y))
    assert bits_equal(outs[0], outs[1])
    ctx.close()


def test_row_split_rejects_bad_threshold(cuda_lib):
    ctx = context(Determinism.kBackendDefault)
    with pytest.raises(AscError) as err:
        ctx.set_variant(Variant.kRowSplit, 3)
    assert err.value.code == ErrorCode.kInvalidArgument
    ctx.close()
