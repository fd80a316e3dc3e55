"""GPU parity of the SpMV entry points against the oracle and the reference's
golden vectors.  Deterministic mode must be bit-exact; BACKEND_DEFAULT
variants must stay inside |y - y_ref| <= gamma_{n+2}(|alpha||A||x| + |beta y|)."""

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import Determinism, ErrorCode, FormatKind, SparseBlasTranspose, Variant
from asc_cpp_b200.sparse_cuda import (AscError, CsrPlan, CudaCsrSpmv,
                                      CudaCsrSpmvWorkspaceSize, CudaSpmv)
from oracle import CSR, OP_NONE, OP_TRANSPOSE

from gpu_util import (assert_within_bound, bits_equal, context, csr, dev, host, vec)

pytestmark = pytest.mark.gpu

DTYPES = [("f64", np.float64), ("f32", np.float32)]


def compat(ctx, a, alpha, x, beta, y, x_stride=1, y_stride=1, x_extent=None, y_extent=None):
    xv = vec(x, x_extent, x_stride, writable=False)
    yv = vec(y, y_extent, y_stride)
    need = CudaCsrSpmvWorkspaceSize(ctx, a, xv, yv)
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda") if need else None
    CudaCsrSpmv(ctx, alpha, a, xv, beta, yv, ws, need)
    return need


@pytest.mark.parametrize("tag,dt", DTYPES)
def test_reference_known_answers(cuda_lib, known_answers, tag, dt):
    ctx = context()
    # sparse_cuda_test.cc:239-352: strided x (2) and y (3), padding untouched
    a = csr(4, 5, [0, 2, 3, 6, 8], [0, 3, 1, 0, 2, 4, 1, 4],
            np.array([2, -1, 4, 7, 3, 5, -2, 6], dt))
    x = dev(np.array([1, 91, -2, 91, 3, 91, 4, 91, -1], dt))
    y = dev(np.array([10, 91, 91, 20, 91, 91, 30, 91, 91, 40], dt))
    need = compat(ctx, a, 2.0, x, -0.5, y, 2, 3, 5, 4)
    assert need == 0  # the strided path takes no workspace (reference rule)
    assert bits_equal(host(y), known_answers[f"cuda_strided_{tag}"])
    yn = dev(np.full(10, np.nan, dt))
    compat(ctx, a, 1.0, x, 0.0, yn, 2, 3, 5, 4)
    assert bits_equal(host(yn), known_answers[f"cuda_strided_beta0_{tag}"])
    # sparse_cuda_test.cc:354-433: unit stride {15, 29}
    a2 = csr(2, 2, [0, 1, 2], [0, 1], np.array([2, 3], dt))
    x2 = dev(np.array([4, 5], dt))
    y2 = dev(np.array([1, 1], dt))
    compat(ctx, a2, 2.0, x2, -1.0, y2)
    assert bits_equal(host(y2), known_answers[f"cuda_unit_{tag}"])
    # blas_test.cc:165-219
    a3 = csr(3, 4, [0, 2, 4, 5], [1, 3, 0, 2, 1], np.array([2, -1, 4, 5, 3], dt))
    x3 = dev(np.array([2, -1, 3, 4], dt))
    y3 = dev(np.array([7, -90, 11, -91, 13, -92], dt))
    compat(ctx, a3, 2.0, x3, -0.5, y3, 1, 2, 4, 3)
    assert bits_equal(host(y3), known_answers[f"blas_compat_a2_bm05_{tag}"])
    # zero columns -> y = beta*y ; empty matrix -> zeros over NaN
    a4 = csr(3, 0, [0, 0, 0, 0], np.zeros(0, np.int64), np.zeros(0, dt))
    y4 = dev(np.array([2, -3, 4], dt))
    compat(ctx, a4, 7.0, dev(np.zeros(1, dt)), 2.0, y4, x_extent=0)
    assert bits_equal(host(y4), known_answers[f"blas_zero_columns_{tag}"])
    a5 = csr(3, 4, [0, 0, 0, 0], np.zeros(0, np.int64), np.zeros(0, dt))
    y5 = dev(np.full(3, np.nan, dt))
    compat(ctx, a5, 1.0, dev(np.zeros(4, dt)), 0.0, y5)
    assert bits_equal(host(y5), known_answers[f"blas_empty_{tag}"])
    ctx.close()


def test_reference_order_known_answer(cuda_lib, known_answers):
    ctx = context()
    a = csr(1, 3, [0, 3], [0, 1, 2], np.array([1e20, 1, -1e20], np.float32))
    y = dev(np.array([-1.0], np.float32))
    compat(ctx, a, 1.0, dev(np.ones(3, np.float32)), 0.0, y)
    out = host(y)
    assert out[0] == 0.0 and bits_equal(out, known_answers["blas_order_f32"])
    ctx.close()


def test_golden_random_cases_bit_exact(cuda_lib, random_cases):
    ctx = context()
    for case in range(int(random_cases["count"][0])):
        p = f"c{case}_"
        rows, cols = (int(v) for v in random_cases[p + "shape"])
        alpha, beta = (float(v) for v in random_cases[p + "ab"])
        a = csr(rows, cols, random_cases[p + "ptr"], random_cases[p + "idx"],
                random_cases[p + "val"])
        y = dev(random_cases[p + "y0"])
        compat(ctx, a, alpha, dev(random_cases[p + "x"]), beta, y)
        assert bits_equal(host(y), random_cases[p + "compat"]), case
        y = dev(random_cases[p + "y0"])
        CudaSpmv(ctx, SparseBlasTranspose.kNone, alpha, a,
                 vec(dev(random_cases[p + "x"]), writable=False), vec(y))
        assert bits_equal(host(y), random_cases[p + "std_none"]), case
    ctx.close()


def test_laplacian_316_bit_exact_against_reference(cuda_lib, laplacian_golden, restatement):
    """Config 1: FP64 y = 1.0*A*x + 0.5*y on the 5-point Laplacian, 316^2 grid."""
    import hashlib
    a_h = synthetic.laplacian_2d(316)
    assert a_h.nnz == 498_016
    rng = np.random.default_rng(0)
    x_h = rng.uniform(-1, 1, a_h.cols)
    y_h = rng.uniform(-1, 1, a_h.rows)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    y = dev(y_h)
    compat(ctx, a, 1.0, dev(x_h), 0.5, y)
    out = host(y)
    assert hashlib.sha256(out.tobytes()).digest() == laplacian_golden["sha256"].tobytes()
    expect = y_h.copy()
    restatement.compat_spmv(a_h.ptr, a_h.idx, a_h.val, 1.0, x_h, 0.5, expect)
    assert bits_equal(out, expect)
    ctx.close()


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("shape", ["irregular", "long_rows", "empty_rows", "single"])
def test_row_ordered_bit_exact_vs_oracle(cuda_lib, restatement, tag, dt, shape):
    rng = np.random.default_rng(hash((tag, shape)) % 2**32)
    if shape == "irregular":
        a_h = synthetic.random_csr(rng, 3000, 2500, 90, dt, 0.1)
    elif shape == "long_rows":
        # rows far longer than the staged window (4096) and tile (2048 items)
        lengths = np.array([1, 9000, 3, 20000, 0, 4097, 2047, 2049, 5000] * 3)
        ptr, idx = synthetic._unique_sorted_rows(rng, 30000, lengths)
        a_h = synthetic.Csr(lengths.size, 30000, ptr, idx,
                            rng.standard_normal(int(ptr[-1])).astype(dt))
    elif shape == "empty_rows":
        a_h = synthetic.random_csr(rng, 20000, 500, 6, dt, 0.9)
    else:
        a_h = synthetic.random_csr(rng, 1, 7, 7, dt)
    x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    for alpha, beta in ((1.0, 0.0), (-1.5, 0.25)):
        y = dev(y0)
        compat(ctx, a, alpha, dev(x_h), beta, y)
        expect = y0.copy()
        restatement.compat_spmv(a_h.ptr, a_h.idx, a_h.val, alpha, x_h, beta, expect)
        assert bits_equal(host(y), expect), (alpha, beta)
        # strided output and input (zero-workspace path, in-kernel tile search)
        xs = np.zeros(a_h.cols * 2, dt)
        xs[::2] = x_h
        ys = np.full(a_h.rows * 3, 7, dt)
        ys[::3] = y0
        yd = dev(ys)
        compat(ctx, a, alpha, dev(xs), beta, yd, 2, 3, a_h.cols, a_h.rows)
        out = host(yd)
        assert bits_equal(out[::3], expect)
        assert np.all(out[1::3] == 7) and np.all(out[2::3] == 7)
        # standard form y += alpha*A*x
        y = dev(y0)
        CudaSpmv(ctx, SparseBlasTranspose.kNone, alpha, a, vec(dev(x_h), writable=False), vec(y))
        expect = y0.copy()
        restatement.standard_spmv(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                                  alpha, x_h, expect)
        assert bits_equal(host(y), expect)
    ctx.close()


def test_plan_path_bit_exact(cuda_lib, restatement):
    rng = np.random.default_rng(11)
    a_h = synthetic.random_csr(rng, 5000, 4000, 60, np.float64, 0.05)
    x_h = rng.uniform(-1, 1, a_h.cols)
    y0 = rng.uniform(-1, 1, a_h.rows)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a)
    y = dev(y0)
    plan.csr_spmv(0.5, vec(dev(x_h), writable=False), 2.0, vec(y))
    expect = y0.copy()
    restatement.compat_spmv(a_h.ptr, a_h.idx, a_h.val, 0.5, x_h, 2.0, expect)
    assert bits_equal(host(y), expect)
    plan.close()
    ctx.close()


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_vector_variant_within_bound(cuda_lib, restatement, tag, dt, lanes):
    rng = np.random.default_rng(lanes)
    a_h = synthetic.random_csr(rng, 4000, 3000, 120, dt, 0.05)
    x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
    ctx = context(Determinism.kBackendDefault)
    ctx.set_variant(Variant.kVector, lanes)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                         a_h.val, x_h)
    counts = np.diff(a_h.ptr)
    alpha, beta = 1.25, -0.5
    y = dev(y0)
    compat(ctx, a, alpha, dev(x_h), beta, y)
    ref = alpha * exact + beta * y0.astype(np.longdouble)
    assert_within_bound(host(y), exact, absval, counts, dt, alpha,
                        np.abs(beta * y0.astype(np.float64)), ref)
    ctx.close()


@pytest.mark.parametrize("tag,dt", DTYPES)
def test_transpose_default_mode_within_bound(cuda_lib, restatement, tag, dt):
    rng = np.random.default_rng(3)
    a_h = synthetic.random_csr(rng, 2000, 1500, 40, dt, 0.1)
    x_h = rng.uniform(-1, 1, a_h.rows).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.cols).astype(dt)
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, 0.75, a, vec(dev(x_h), writable=False), vec(y))
    exact, absval = restatement.extended(OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                         a_h.val, x_h)
    counts = restatement.output_counts(OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx)
    ref = y0.astype(np.longdouble) + 0.75 * exact
    assert_within_bound(host(y), exact, absval, counts, dt, 0.75,
                        np.abs(y0.astype(np.float64)), ref)
    # CSC with op = none is the same product on the same arrays
    c = csr(a_h.cols, a_h.rows, a_h.ptr, a_h.idx, a_h.val, FormatKind.kCsc)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 0.75, c, vec(dev(x_h), writable=False), vec(y))
    assert_within_bound(host(y), exact, absval, counts, dt, 0.75,
                        np.abs(y0.astype(np.float64)), ref)
    ctx.close()


def test_csc_transpose_is_row_ordered_bit_exact(cuda_lib, restatement):
    """CSC with op = transpose reads the arrays as CSR rows: bit-exact."""
    from oracle import CSC
    rng = np.random.default_rng(8)
    a_h = synthetic.random_csr(rng, 700, 900, 30, np.float64, 0.1)  # arrays = CSC of 900x700
    x_h = rng.uniform(-1, 1, a_h.cols)
    y0 = rng.uniform(-1, 1, a_h.rows)
    ctx = context()
    c = csr(a_h.cols, a_h.rows, a_h.ptr, a_h.idx, a_h.val, FormatKind.kCsc)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, -2.0, c, vec(dev(x_h), writable=False), vec(y))
    expect = y0.copy()
    restatement.standard_spmv(CSC, OP_TRANSPOSE, a_h.cols, a_h.rows, a_h.ptr, a_h.idx, a_h.val,
                              -2.0, x_h, expect)
    assert bits_equal(host(y), expect)
    ctx.close()


def test_negative_strides_standard(cuda_lib, restatement):
    rng = np.random.default_rng(9)
    a_h = synthetic.random_csr(rng, 300, 200, 20, np.float64, 0.1)
    x_store = rng.uniform(-1, 1, 2 * a_h.cols)
    y_store = rng.uniform(-1, 1, a_h.rows)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    y = dev(y_store)
    xv = vec(dev(x_store), a_h.cols, -2, 2 * (a_h.cols - 1), writable=False)
    yv = vec(y, a_h.rows, -1, a_h.rows - 1)
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 1.5, a, xv, yv)
    expect = y_store.copy()
    restatement.standard_spmv(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val, 1.5,
                              x_store, expect, incx=-2, incy=-1, x_offset=2 * (a_h.cols - 1),
                              y_offset=a_h.rows - 1)
    assert bits_equal(host(y), expect)
    ctx.close()


def test_alpha_zero_reads_nothing(cuda_lib):
    """blas.h:1650-1652: alpha == 0 leaves y untouched even with NaN values."""
    ctx = context()
    a = csr(2, 2, [0, 1, 3], [0, 0, 1], np.full(3, np.nan))
    y = dev(np.array([7.0, 9.0]))
    CudaSpmv(ctx, SparseBlasTranspose.kNone, 0.0, a, vec(dev(np.array([1.0, -1.0])),
                                                         writable=False), vec(y))
    assert list(host(y)) == [7.0, 9.0]
    ctx.close()


def test_failures_do_not_mutate(cuda_lib):
    ctx = context()
    a = csr(3, 4, [0, 2, 4, 5], [1, 3, 0, 2, 1], np.array([2, -1, 4, 5, 3.0]))
    x = dev(np.array([2, -1, 3, 4.0]))
    y = dev(np.array([1, 2, 3.0]))
    before = host(y).copy()
    # wrong output length
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0, vec(y, 2), None, 0)
    assert e.value.code == ErrorCode.kShape
    # output overlapping the input
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0, vec(x, 3), None, 0)
    assert e.value.code == ErrorCode.kInvalidArgument
    # host memory
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0,
                    vec(torch.zeros(3, dtype=torch.float64)), None, 0)
    assert e.value.code == ErrorCode.kMemoryAccess
    # workspace too small / host workspace on the unit-stride path
    need = CudaCsrSpmvWorkspaceSize(ctx, a, vec(x, writable=False), vec(y))
    assert need > 0
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0, vec(y), ws, need - 1)
    assert e.value.code == ErrorCode.kInvalidArgument
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0, vec(y),
                    torch.empty(need, dtype=torch.uint8), need)
    assert e.value.code == ErrorCode.kInvalidArgument
    # a strided call with a workspace is rejected
    y9 = dev(np.zeros(9))
    with pytest.raises(AscError) as e:
        CudaCsrSpmv(ctx, 1.0, a, vec(x, writable=False), 0.0, vec(y9, 3, 3), ws, need)
    assert e.value.code == ErrorCode.kInvalidArgument
    assert not host(y9).any()
    # untrusted structure
    d = a.describe()
    d.canonical_structure_trusted = 0
    import ctypes
    xd, yd = vec(x, writable=False).describe(), vec(y).describe()
    rc = ctx._lib.asc_sb_csr_spmv(ctx.handle, 1.0, ctypes.byref(d), ctypes.byref(xd), 0.0,
                                  ctypes.byref(yd), None, 0, 2)
    assert rc == ErrorCode.kInvalidArgument
    assert bits_equal(host(y), before)
    ctx.close()


def _shapes(rng, dt):
    lengths = np.array([1, 9000, 3, 20000, 0, 4097, 2047, 2049, 5000, 0, 0, 257, 255, 256] * 2)
    ptr, idx = synthetic._unique_sorted_rows(rng, 30000, lengths)
    long_rows = synthetic.Csr(lengths.size, 30000, ptr, idx,
                              rng.standard_normal(int(ptr[-1])).astype(dt))
    # rows of 0..8 and 240..255 entries: tiles whose window starts up to 7
    # positions before their first row and whose second row starts ~250
    # positions later (the edge of the 256-position window)
    lead = np.where(rng.random(20000) < 0.5, rng.integers(0, 9, 20000),
                    rng.integers(240, 256, 20000))
    lptr, lidx = synthetic._unique_sorted_rows(rng, 30000, lead)
    return {
        "window_leads": synthetic.Csr(lead.size, 30000, lptr, lidx,
                                      rng.standard_normal(int(lptr[-1])).astype(dt)),
        "irregular": synthetic.random_csr(rng, 3000, 2500, 90, dt, 0.1),
        "long_rows": long_rows,
        "empty_rows": synthetic.random_csr(rng, 20000, 500, 6, dt, 0.9),
        "power_law": synthetic.power_law(20000, seed=5, dtype=dt),
        "single": synthetic.random_csr(rng, 1, 7, 7, dt),
    }


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("misalign", [False, True])
def test_merge_variant_within_bound(cuda_lib, restatement, tag, dt, misalign):
    """MERGE_PATH (contracted: the merge partition on the segmented tile
    body; the scalar-load kernel when the arrays are not 16-byte aligned)
    stays inside the error bound on every shape."""
    rng = np.random.default_rng(21)
    ctx = context(Determinism.kBackendDefault)
    ctx.set_variant(Variant.kMergePath)
    for name, a_h in _shapes(rng, dt).items():
        x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
        y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        if misalign:  # idx/val views starting 8 (resp. 4) bytes into a buffer
            idx_store = torch.zeros(a_h.nnz + 1, dtype=torch.int64, device="cuda")
            val_store = torch.zeros(a_h.nnz + 1, dtype=a.values.dtype, device="cuda")
            idx_store[1:] = a.indices
            val_store[1:] = a.values
            a.indices, a.values = idx_store[1:], val_store[1:]
        exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                             a_h.val, x_h)
        counts = np.diff(a_h.ptr)
        for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
            y = dev(y0)
            compat(ctx, a, alpha, dev(x_h), beta, y)
            ref = alpha * exact + beta * y0.astype(np.longdouble)
            assert_within_bound(host(y), exact, absval, counts, dt, alpha,
                                np.abs(beta * y0.astype(np.float64)), ref)
            y = dev(y0)
            CudaSpmv(ctx, SparseBlasTranspose.kNone, alpha, a, vec(dev(x_h), writable=False),
                     vec(y))
            ref = y0.astype(np.longdouble) + alpha * exact
            assert_within_bound(host(y), exact, absval, counts, dt, alpha,
                                np.abs(y0.astype(np.float64)), ref)
    assert ctx.device_status() == 0
    ctx.close()


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("misalign", [False, True])
def test_warp_tiles_variant_within_bound(cuda_lib, restatement, tag, dt, misalign):
    """WARP_TILES (register-segmented kernel; scalar-load kernel when the
    arrays are not 16-byte aligned) stays inside the error bound."""
    rng = np.random.default_rng(23)
    ctx = context(Determinism.kBackendDefault)
    ctx.set_variant(Variant.kWarpTiles)
    for name, a_h in _shapes(rng, dt).items():
        x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
        y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        if misalign:  # idx/val views starting 8 (resp. 4) bytes into a buffer
            idx_store = torch.zeros(a_h.nnz + 1, dtype=torch.int64, device="cuda")
            val_store = torch.zeros(a_h.nnz + 1, dtype=a.values.dtype, device="cuda")
            idx_store[1:] = a.indices
            val_store[1:] = a.values
            a.indices, a.values = idx_store[1:], val_store[1:]
        exact, absval = restatement.extended(OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                             a_h.val, x_h)
        counts = np.diff(a_h.ptr)
        for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
            y = dev(y0)
            compat(ctx, a, alpha, dev(x_h), beta, y)
            ref = alpha * exact + beta * y0.astype(np.longdouble)
            assert_within_bound(host(y), exact, absval, counts, dt, alpha,
                                np.abs(beta * y0.astype(np.float64)), ref)
            y = dev(y0)
            CudaSpmv(ctx, SparseBlasTranspose.kNone, alpha, a, vec(dev(x_h), writable=False),
                     vec(y))
            ref = y0.astype(np.longdouble) + alpha * exact
            assert_within_bound(host(y), exact, absval, counts, dt, alpha,
                                np.abs(y0.astype(np.float64)), ref)
    ctx.close()


@pytest.mark.parametrize("tag,dt", DTYPES)
@pytest.mark.parametrize("misalign", [False, True])
def test_exact_paths_bit_exact_on_all_shapes(cuda_lib, restatement, tag, dt, misalign):
    """Deterministic mode through every route: workspace partition, no
    partition (in-kernel tile search), plan; 16-byte aligned arrays take the
    register-segmented kernel, misaligned ones the scalar-load warp kernel."""
    rng = np.random.default_rng(22)
    ctx = context()
    for name, a_h in _shapes(rng, dt).items():
        x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
        y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
        a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
        if misalign:
            idx_store = torch.zeros(a_h.nnz + 1, dtype=torch.int64, device="cuda")
            val_store = torch.zeros(a_h.nnz + 1, dtype=a.values.dtype, device="cuda")
            idx_store[1:] = a.indices
            val_store[1:] = a.values
            a.indices, a.values = idx_store[1:], val_store[1:]
        expect = y0.copy()
        restatement.compat_spmv(a_h.ptr, a_h.idx, a_h.val, 1.25, x_h, -0.5, expect)
        y = dev(y0)
        compat(ctx, a, 1.25, dev(x_h), -0.5, y)
        assert bits_equal(host(y), expect), name
        plan = CsrPlan(ctx, a)
        y = dev(y0)
        plan.csr_spmv(1.25, vec(dev(x_h), writable=False), -0.5, vec(y))
        assert bits_equal(host(y), expect), name
        expect_std = y0.copy()
        restatement.standard_spmv(CSR, OP_NONE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                                  -2.0, x_h, expect_std)
        y = dev(y0)
        CudaSpmv(ctx, SparseBlasTranspose.kNone, -2.0, a, vec(dev(x_h), writable=False), vec(y),
                 plan=plan)
        assert bits_equal(host(y), expect_std), name
        y = dev(y0)
        CudaSpmv(ctx, SparseBlasTranspose.kNone, -2.0, a, vec(dev(x_h), writable=False), vec(y))
        assert bits_equal(host(y), expect_std), name
        plan.close()
    assert ctx.device_status() == 0
    ctx.close()
