"""GPU parity of the sparse triangular solve (asc_sb_standard_triangular_solve,
the replacement of internal_sparse_cuda::StandardTriangularSolveErased, and
asc_sb_plan_triangular_solve): the reference's own outputs
(tests/golden/trsv_cases.npz), bit-identical DETERMINISTIC solves against the
oracle at sizes up to 10^6 rows, BACKEND_DEFAULT within tolerance and
reproducible, plans, empty operands and the validation failures of
operations.cc:1380-1436."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import (PLAN_TRANSPOSE, PLAN_TRIANGULAR, Determinism, ErrorCode,
                               FormatKind, SparseBlasDiagonal, SparseBlasLayout,
                               SparseBlasTranspose, SparseBlasTriangle)
from asc_cpp_b200.sparse_cuda import (AscError, CsrPlan, CudaSparseTriangularSolve,
                                      CudaSparseTriangularSolveMultiple, DenseMatrixView)

from gpu_util import bits_equal, context, csr, dev, host, vec
from test_oracle import TRSV_SHAPES, TRSV_TAGS, trsv_fixture_cases

pytestmark = pytest.mark.gpu

OPS = (SparseBlasTranspose.kNone, SparseBlasTranspose.kTranspose,
       SparseBlasTranspose.kConjugateTranspose)


def _dense(t, n, k, layout):
    return DenseMatrixView(t, n, k, SparseBlasLayout(layout))


def _solve(ctx, op, alpha, a, tri, diag, b_host, n, k, layout, plan=None):
    b = dev(b_host)
    CudaSparseTriangularSolveMultiple(ctx, op, alpha, a, tri, diag, _dense(b, n, k, layout),
                                      plan=plan)
    return host(b)


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_reference_fixtures(cuda_lib, restatement, trsv_cases, tag):
    """Bit-identical to the reference's solves; complex FP32 with a non-unit
    diagonal is bit-identical to the oracle's Smith division (the facet's)
    and within a few ulps of the reference's libgcc division."""
    ctx = context()
    for (key, op, tri, diag, layout, k, alpha, ptr, idx, val, b,
         x) in trsv_fixture_cases(trsv_cases, tag):
        a = csr(48, 48, ptr, idx, val)
        got = _solve(ctx, op, alpha, a, tri, diag, b, 48, k, layout)
        if tag == "c" and diag == 0:
            want = restatement.triangular_solve(op, tri, diag, 48, ptr, idx, val, alpha, b,
                                                layout, None, k)
            assert bits_equal(got, want), key
            np.testing.assert_allclose(got, x, rtol=2e-5, atol=2e-6, err_msg=key)
        else:
            assert bits_equal(got, x), key
    ctx.close()


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_known_answers(cuda_lib, trsv_cases, tag):
    """standard_blas_cuda_test.cc:542-680 through the vector and multiple
    entry points."""
    g = trsv_cases
    ctx = context()
    ptr = np.array([0, 1, 3], np.int64)
    idx = np.array([0, 0, 1], np.int64)
    a = csr(2, 2, ptr, idx, g[f"ka_{tag}_val"])
    lower, nonunit = SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit
    for name, op in (("vec", SparseBlasTranspose.kNone),
                     ("ct", SparseBlasTranspose.kConjugateTranspose)):
        b = dev(g[f"ka_{name}_{tag}_b"])
        CudaSparseTriangularSolve(ctx, op, 1.0, a, lower, nonunit, vec(b))
        assert bits_equal(host(b), g[f"ka_{name}_{tag}_x"])
    got = _solve(ctx, SparseBlasTranspose.kNone, 1.0, a, lower, nonunit,
                 g[f"ka_multi_{tag}_b"], 2, 2, 1)
    assert bits_equal(got, g[f"ka_multi_{tag}_x"])
    z = csr(2, 2, ptr, idx, g[f"ka_zero_{tag}_val"])
    b = dev(np.array([4, 5], g[f"ka_zero_{tag}_val"].dtype))
    CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 0.0, z, lower, nonunit, vec(b))
    assert bits_equal(host(b), g[f"ka_zero_{tag}_x"])
    if f"ka_large_{tag}_val" in g:
        lv = g[f"ka_large_{tag}_val"]
        one = csr(1, 1, np.array([0, 1], np.int64), np.array([0], np.int64), lv)
        b = dev(lv)
        CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 1.0, one, lower, nonunit,
                                  vec(b))
        assert bits_equal(host(b), g[f"ka_large_{tag}_x"])
    ctx.close()


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_large_deterministic_bit_exact(cuda_lib, restatement, tag):
    """200k rows, every triangle / op / diagonal, one and four right-hand
    sides in both layouts: bit-identical to the oracle."""
    dt = TRSV_TAGS[tag]
    rng = np.random.default_rng(31)
    n = 200_000
    ctx = context()
    cplx = np.iscomplexobj(dt(0))
    alpha = (1.25 + 0.5j) if cplx else 1.25
    for tri in (SparseBlasTriangle.kLower, SparseBlasTriangle.kUpper):
        m = synthetic.triangular(rng, n, lower=tri == SparseBlasTriangle.kLower, near=4, far=2,
                                 span=200, dtype=dt)
        # with a unit diagonal the stored one is ignored: smaller entries keep
        # the solution finite (NaN payloads are not compared bit for bit)
        small = (m.val * dt(0.1)).astype(dt)
        for diag in (SparseBlasDiagonal.kNonUnit, SparseBlasDiagonal.kUnit):
            val = m.val if diag == SparseBlasDiagonal.kNonUnit else small
            a = csr(n, n, m.ptr, m.idx, val)
            for op in OPS:
                for layout, k in ((1, 1), (1, 4), (0, 4)):
                    if k > 1 and (op != SparseBlasTranspose.kNone
                                  and diag == SparseBlasDiagonal.kUnit):
                        continue
                    b = synthetic._values(rng, n * k, dt)
                    got = _solve(ctx, op, alpha, a, tri, diag, b, n, k, layout)
                    want = restatement.triangular_solve(int(op), int(tri), int(diag), n, m.ptr,
                                                        m.idx, val, alpha, b, layout, None, k)
                    assert np.isfinite(want).all()
                    assert bits_equal(got, want), (tri, op, diag, layout, k)
    status = ctypes.c_int32()
    ctx.check(ctx._lib.asc_sb_context_device_status(ctx.handle, ctypes.byref(status), 1))
    assert status.value == 0
    ctx.close()


def test_million_row_chain_and_laplacian(cuda_lib, restatement):
    """Long dependency chains: a bidiagonal matrix of 10^6 rows (every row
    waits for the previous one) and the lower triangle of a 1000 x 1000
    5-point Laplacian (1999 wavefronts)."""
    n = 1_000_000
    ptr = np.concatenate([[0], np.arange(1, 2 * n, 2)]).astype(np.int64)
    idx = np.empty(2 * n - 1, np.int64)
    idx[0] = 0
    idx[1::2] = np.arange(0, n - 1)
    idx[2::2] = np.arange(1, n)
    rng = np.random.default_rng(5)
    val = rng.uniform(0.5, 1.0, 2 * n - 1)
    val[0] = 2.0
    val[2::2] = rng.uniform(2.0, 3.0, n - 1)
    b = rng.uniform(-1, 1, n)
    ctx = context()
    got = _solve(ctx, SparseBlasTranspose.kNone, 1.0, csr(n, n, ptr, idx, val),
                 SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit, b, n, 1, 1)
    want = restatement.triangular_solve(0, 1, 0, n, ptr, idx, val, 1.0, b)
    assert bits_equal(got, want)
    lap = synthetic.triangle_of(synthetic.laplacian_2d(1000))
    b = rng.uniform(-1, 1, lap.rows)
    got = _solve(ctx, SparseBlasTranspose.kNone, -0.5, csr(lap.rows, lap.cols, lap.ptr, lap.idx,
                                                           lap.val),
                 SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit, b, lap.rows, 1, 1)
    want = restatement.triangular_solve(0, 1, 0, lap.rows, lap.ptr, lap.idx, lap.val, -0.5, b)
    assert bits_equal(got, want)
    ctx.close()


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_backend_default_close_and_reproducible(cuda_lib, restatement, tag):
    dt = TRSV_TAGS[tag]
    rng = np.random.default_rng(37)
    n = 300_000
    m = synthetic.triangular(rng, n, lower=True, near=12, far=4, span=500, dtype=dt)
    a = csr(n, n, m.ptr, m.idx, m.val)
    b = synthetic._values(rng, n, dt)
    ctx = context(Determinism.kBackendDefault)
    runs = [_solve(ctx, op, 1.0, a, SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit,
                   b, n, 1, 1) for op in (SparseBlasTranspose.kNone,) * 3]
    assert all(bits_equal(r, runs[0]) for r in runs[1:])
    want = restatement.triangular_solve(0, 1, 0, n, m.ptr, m.idx, m.val, 1.0, b)
    tol = 1e-12 if dt in (np.float64, np.complex128) else 2e-5
    assert np.max(np.abs(runs[0] - want)) <= tol * max(1.0, np.max(np.abs(want)))
    ctx.close()


def test_plan_solves_match_unplanned(cuda_lib, restatement):
    rng = np.random.default_rng(43)
    n = 50_000
    ctx = context()
    m = synthetic.triangular(rng, n, lower=False, dtype=np.float64)
    a = csr(n, n, m.ptr, m.idx, m.val)
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE | PLAN_TRIANGULAR)
    for op in OPS:
        b = rng.uniform(-1, 1, n * 3)
        got = _solve(ctx, op, 0.75, a, SparseBlasTriangle.kUpper, SparseBlasDiagonal.kNonUnit,
                     b, n, 3, 0, plan=plan)
        want = _solve(ctx, op, 0.75, a, SparseBlasTriangle.kUpper, SparseBlasDiagonal.kNonUnit,
                      b, n, 3, 0)
        assert bits_equal(got, want)
        assert bits_equal(got, restatement.triangular_solve(int(op), 0, 0, n, m.ptr, m.idx, m.val,
                                                            0.75, b, 0, None, 3))
    plan.close()
    # a plan without triangular state, or without the transposed structure
    plain = CsrPlan(ctx, a)
    with pytest.raises(AscError) as e:
        _solve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kUpper,
               SparseBlasDiagonal.kUnit, np.ones(n), n, 1, 1, plan=plain)
    assert e.value.code == ErrorCode.kInvalidState
    plain.close()
    tri_only = CsrPlan(ctx, a, PLAN_TRIANGULAR)
    with pytest.raises(AscError) as e:
        _solve(ctx, SparseBlasTranspose.kTranspose, 1.0, a, SparseBlasTriangle.kUpper,
               SparseBlasDiagonal.kUnit, np.ones(n), n, 1, 1, plan=tri_only)
    assert e.value.code == ErrorCode.kInvalidState
    tri_only.close()
    ctx.close()


@pytest.mark.parametrize("det", [Determinism.kDeterministic, Determinism.kBackendDefault])
def test_level_order_analysis(cuda_lib, restatement, det):
    """After asc_sb_plan_triangular_analysis the plan's solves run in level
    order and give the same bits as the row-order solve, for matching and
    for mismatching (ignored) analyses, one and three right-hand sides."""
    rng = np.random.default_rng(53)
    ctx = context(det)
    lap = synthetic.triangle_of(synthetic.laplacian_2d(300))
    rand = synthetic.triangular(rng, 100_000, lower=True, near=3, far=3, span=5000,
                                dtype=np.complex128)
    for m in (lap, rand):
        n = m.rows
        a = csr(n, n, m.ptr, m.idx, m.val)
        plan = CsrPlan(ctx, a, PLAN_TRANSPOSE | PLAN_TRIANGULAR)
        for op, tri in ((SparseBlasTranspose.kNone, SparseBlasTriangle.kLower),
                        (SparseBlasTranspose.kConjugateTranspose, SparseBlasTriangle.kLower)):
            for k, layout in ((1, 1), (3, 0)):
                b = synthetic._values(rng, n * k, m.val.dtype)
                want = _solve(ctx, op, 1.5, a, tri, SparseBlasDiagonal.kNonUnit, b, n, k, layout)
                plan.triangular_analysis(op, tri)
                got = _solve(ctx, op, 1.5, a, tri, SparseBlasDiagonal.kNonUnit, b, n, k, layout,
                             plan=plan)
                assert bits_equal(got, want), (op, k)
                if det == Determinism.kDeterministic:
                    ref = restatement.triangular_solve(int(op), int(tri), 0, n, m.ptr, m.idx,
                                                       m.val, 1.5, b, layout, None, k)
                    assert bits_equal(got, ref)
        # an analysis of the other op class is not used, and nothing changes
        plan.triangular_analysis(SparseBlasTranspose.kTranspose, SparseBlasTriangle.kLower)
        b = synthetic._values(rng, n, m.val.dtype)
        assert bits_equal(_solve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kLower,
                                 SparseBlasDiagonal.kNonUnit, b, n, 1, 1, plan=plan),
                          _solve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kLower,
                                 SparseBlasDiagonal.kNonUnit, b, n, 1, 1))
        plan.close()
    ctx.close()


def test_strided_vector_and_padding(cuda_lib, restatement):
    """A vector with increment 3 (the reference's vector binding): only its
    elements change; the padding between them is never written."""
    rng = np.random.default_rng(47)
    n = 20_000
    m = synthetic.triangular(rng, n, lower=True, dtype=np.float32)
    full = rng.uniform(-1, 1, 3 * n + 2).astype(np.float32)
    t = dev(full)
    ctx = context()
    CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 2.0, csr(n, n, m.ptr, m.idx, m.val),
                              SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit,
                              vec(t, extent=n, stride=3, offset=1))
    got = host(t)
    want = restatement.triangular_solve(0, 1, 0, n, m.ptr, m.idx, m.val, 2.0,
                                        full[1::3][:n].copy())
    assert bits_equal(got[1::3][:n].copy(), want)
    pad = np.ones(full.size, bool)
    pad[1:1 + 3 * n:3] = False
    assert bits_equal(got[pad], full[pad])
    ctx.close()


def test_empty_operands(cuda_lib):
    ctx = context()
    a0 = csr(0, 0, np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0))
    t = torch.zeros(0, dtype=torch.float64, device="cuda")
    CudaSparseTriangularSolveMultiple(ctx, SparseBlasTranspose.kNone, 1.0, a0,
                                      SparseBlasTriangle.kLower, SparseBlasDiagonal.kUnit,
                                      DenseMatrixView(t, 0, 3))
    a = csr(3, 3, np.array([0, 1, 2, 3], np.int64), np.arange(3, dtype=np.int64), np.ones(3))
    CudaSparseTriangularSolveMultiple(ctx, SparseBlasTranspose.kNone, 1.0, a,
                                      SparseBlasTriangle.kLower, SparseBlasDiagonal.kUnit,
                                      DenseMatrixView(t, 3, 0))
    ctx.close()


def test_validation_failures(cuda_lib):
    """operations.cc:1380-1436: enums, square CSR only, extents, writability,
    overlap of the right-hand sides with the matrix; nothing is written."""
    ctx = context()
    n = 4
    ptr = np.array([0, 1, 2, 3, 4], np.int64)
    idx = np.arange(4, dtype=np.int64)
    a = csr(n, n, ptr, idx, np.full(4, 2.0))
    b0 = np.arange(1.0, 5.0)
    lower, unit = SparseBlasTriangle.kLower, SparseBlasDiagonal.kUnit

    def code(fn):
        with pytest.raises(AscError) as e:
            fn()
        return e.value.code

    b = dev(b0)
    view = DenseMatrixView(b, n, 1)
    solve = CudaSparseTriangularSolveMultiple
    assert code(lambda: solve(ctx, 7, 1.0, a, lower, unit, view)) == ErrorCode.kInvalidArgument
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a, 5, unit,
                              view)) == ErrorCode.kInvalidArgument
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a, lower, 9,
                              view)) == ErrorCode.kInvalidArgument
    csc = csr(n, n, ptr, idx, np.full(4, 2.0), FormatKind.kCsc)
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, csc, lower, unit,
                              view)) == ErrorCode.kShape
    rect = csr(n, n + 1, ptr, idx, np.full(4, 2.0))
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, rect, lower, unit,
                              view)) == ErrorCode.kShape
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a, lower, unit,
                              DenseMatrixView(b, n - 1, 1))) == ErrorCode.kShape
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a, lower, unit,
                              DenseMatrixView(b, n, 1, writable=False))) \
        == ErrorCode.kInvalidArgument
    f32 = dev(b0.astype(np.float32))
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a, lower, unit,
                              DenseMatrixView(f32, n, 1))) == ErrorCode.kInvalidArgument
    # right-hand sides inside the matrix's value array
    vals = dev(np.full(8, 2.0))
    a_alias = csr(n, n, ptr, idx, np.full(4, 2.0))
    a_alias.values = vals[:4]
    assert code(lambda: solve(ctx, SparseBlasTranspose.kNone, 1.0, a_alias, lower, unit,
                              DenseMatrixView(vals[2:6], n, 1))) == ErrorCode.kInvalidArgument
    assert bits_equal(host(b), b0)
    ctx.close()
