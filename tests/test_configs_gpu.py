"""GPU parity at the full sizes of the measured configurations, against the
CPU oracle on the same seeded inputs:

* the 4,194,304-row lognormal power-law matrix (row lengths mean 16, sigma
  1.5, clipped to [1, 65536], seed 1), FP64 and FP32, y = A x + beta y and
  the transposed product y += A^T x;
* the 27-point stencil on a 128^3 grid (2,097,152 rows), FP32 C = A B with
  k = 8, 32, 128 row-major right-hand sides (seed 2);
* the 65,536-row matrix of dense 16 x 16 blocks at 2% block density, FP32,
  the same k, through the tensor-core plan;
* the batch of 4096 banded FP64 matrices (seed 3), one graph-captured
  persistent launch.

DETERMINISTIC results must equal the oracle bit for bit.  BACKEND_DEFAULT
results must satisfy |y - y_ref| <= gamma_{n+2}(|alpha| sum|a x| + |beta y0|)
with y_ref the oracle in long double (FP64 data) or in FP64 (FP32 data; the
FP64 oracle's own gamma_{n+2} error is added to the bound).  The oracle runs
on row blocks in parallel threads; per row it is the serial restatement."""

import numpy as np
import pytest
import torch

import oracle
from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import (PLAN_HAS_BLOCKS16, PLAN_HAS_STAGED_SPMM, PLAN_ROW_GROUPS,
                               PLAN_TRANSPOSE, Determinism,
                               SparseBlasTranspose, Variant)
from asc_cpp_b200.sparse_cuda import (CsrPlan, CudaBatch, CudaCsrArray, CudaCsrSpmv,
                                      CudaCsrSpmvWorkspaceSize, CudaSpmm, CudaSpmv,
                                      CudaStridedVectorView, DenseMatrixView)
from oracle import CSR, OP_NONE, OP_TRANSPOSE

from gpu_util import bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu

_CACHE = {}


def power_law_4m(dtype):
    if "pl" not in _CACHE:
        _CACHE["pl"] = synthetic.power_law(4_194_304, 16.0, 1.5, 65_536, seed=1,
                                           dtype=np.float64)
    a = _CACHE["pl"]
    return a if dtype == np.float64 else a.astype(dtype)


def compat(ctx, a, alpha, x, beta, y):
    xv, yv = vec(x, writable=False), vec(y)
    need = CudaCsrSpmvWorkspaceSize(ctx, a, xv, yv)
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    CudaCsrSpmv(ctx, alpha, a, xv, beta, yv, ws, need)


def check_report(rep, what):
    assert rep["max_ratio_to_bound"] <= 1.0, (what, rep)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["f64", "f32"])
def test_powerlaw_4m_spmv(cuda_lib, restatement, dt):
    a_h = power_law_4m(dt)
    assert a_h.rows == 4_194_304 and a_h.nnz == 67_425_776
    rng = np.random.default_rng(1001)
    x_h = rng.uniform(-1, 1, a_h.cols).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.rows).astype(dt)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    x = dev(x_h)
    for alpha, beta in ((1.0, 0.0), (1.0, 0.5)):
        want = oracle.compat_spmv_rows(restatement, a_h.ptr, a_h.idx, a_h.val, alpha, x_h, beta,
                                       y0.copy())
        y = dev(y0)
        compat(ctx, a, alpha, x, beta, y)
        assert bits_equal(host(y), want), (alpha, beta)
        plan = CsrPlan(ctx, a)
        y = dev(y0)
        plan.csr_spmv(alpha, vec(x, writable=False), beta, vec(y))
        assert bits_equal(host(y), want), ("plan", alpha, beta)
        plan.close()
    # BACKEND_DEFAULT: every variant within the bound
    exact, absval = oracle.extended_rows(restatement, a_h.cols, a_h.ptr, a_h.idx, a_h.val, x_h)
    counts = np.diff(a_h.ptr)
    alpha, beta = 1.0, 0.5
    ref = alpha * exact + beta * y0.astype(np.longdouble)
    ctx.set_determinism(Determinism.kBackendDefault)
    for variant, lanes in ((Variant.kAuto, 0), (Variant.kWarpTiles, 0), (Variant.kMergePath, 0),
                           (Variant.kVector, 8), (Variant.kRowSplit, 0)):
        ctx.set_variant(variant, lanes)
        y = dev(y0)
        compat(ctx, a, alpha, x, beta, y)
        rep = oracle.error_report(host(y), ref, absval, counts, dt, alpha,
                                  np.abs(beta * y0.astype(np.float64)))
        check_report(rep, (variant, lanes))
    assert ctx.device_status() == 0
    ctx.close()


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["f64", "f32"])
def test_powerlaw_4m_transposed_spmv(cuda_lib, restatement, dt):
    """y += alpha * A^T x on the full matrix: DETERMINISTIC through a
    transpose plan bit for bit, BACKEND_DEFAULT with and without the plan
    within the bound."""
    a_h = power_law_4m(dt)
    rng = np.random.default_rng(1002)
    x_h = rng.uniform(-1, 1, a_h.rows).astype(dt)
    y0 = rng.uniform(-1, 1, a_h.cols).astype(dt)
    alpha = -0.75
    want = y0.copy()
    restatement.standard_spmv(CSR, OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val,
                              alpha, x_h, want)
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    x = dev(x_h)
    plan = CsrPlan(ctx, a, PLAN_TRANSPOSE)
    y = dev(y0)
    CudaSpmv(ctx, SparseBlasTranspose.kTranspose, alpha, a, vec(x, writable=False), vec(y),
             plan=plan)
    assert bits_equal(host(y), want)
    exact, absval = restatement.extended(OP_TRANSPOSE, a_h.rows, a_h.cols, a_h.ptr, a_h.idx,
                                         a_h.val, x_h)
    counts = np.bincount(a_h.idx, minlength=a_h.cols)
    ref = y0.astype(np.longdouble) + alpha * exact
    ctx.set_determinism(Determinism.kBackendDefault)
    for use_plan in (True, False):
        y = dev(y0)
        CudaSpmv(ctx, SparseBlasTranspose.kTranspose, alpha, a, vec(x, writable=False), vec(y),
                 plan=plan if use_plan else None)
        rep = oracle.error_report(host(y), ref, absval, counts, dt, alpha,
                                  np.abs(y0.astype(np.float64)))
        check_report(rep, ("plan" if use_plan else "scatter"))
    plan.close()
    assert ctx.device_status() == 0
    ctx.close()


def spmm_default_check(restatement, a_h, b, got, alpha, bound_fn, chunk=32):
    """BACKEND_DEFAULT SpMM (C0 = 0) against the FP64 oracle on the same
    FP32 inputs, column block by column block; bound_fn(counts, absval)
    gives the allowed error per output."""
    a64 = a_h.val.astype(np.float64)
    aabs = np.abs(a64)
    counts = np.diff(a_h.ptr)[:, None]
    worst = 0.0
    for j0 in range(0, b.shape[1], chunk):
        j1 = min(b.shape[1], j0 + chunk)
        b64 = np.ascontiguousarray(b[:, j0:j1], dtype=np.float64)
        ref = oracle.standard_spmm_rows(restatement, a_h.cols, a_h.ptr, a_h.idx, a64, alpha, b64,
                                        np.zeros((a_h.rows, j1 - j0)))
        absval = oracle.standard_spmm_rows(restatement, a_h.cols, a_h.ptr, a_h.idx, aabs, 1.0,
                                           np.abs(b64), np.zeros((a_h.rows, j1 - j0)))
        bound = (bound_fn(counts, abs(alpha) * absval) +
                 oracle.gamma(counts + 2, np.float64) * abs(alpha) * absval +
                 np.finfo(np.float32).tiny)
        err = np.abs(got[:, j0:j1].astype(np.float64) - ref)
        ratio = float(np.max(err / bound))
        assert ratio <= 1.0, (j0, ratio)
        worst = max(worst, ratio)
    return worst


def run_spmm(ctx, a, b_d, rows, cols, k, alpha, plan=None):
    c = torch.zeros((rows, k), dtype=torch.float32, device="cuda")
    CudaSpmm(ctx, SparseBlasTranspose.kNone, alpha, a,
             DenseMatrixView(b_d, cols, k, writable=False), DenseMatrixView(c, rows, k),
             plan=plan)
    return host(c)


@pytest.mark.parametrize("k", [8, 32, 128])
def test_stencil_128_spmm(cuda_lib, restatement, k):
    if "st" not in _CACHE:
        _CACHE["st"] = synthetic.stencil_27(128, seed=2, dtype=np.float32)
    a_h = _CACHE["st"]
    assert a_h.rows == 2_097_152 and a_h.nnz == 55_742_968
    rng = np.random.default_rng(2)
    b = rng.standard_normal((a_h.cols, k), dtype=np.float32)
    alpha = 1.0
    ctx = context()
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    b_d = dev(b)
    got = run_spmm(ctx, a, b_d, a_h.rows, a_h.cols, k, alpha)
    want = oracle.standard_spmm_rows(restatement, a_h.cols, a_h.ptr, a_h.idx, a_h.val, alpha, b,
                                     np.zeros((a_h.rows, k), np.float32))
    assert bits_equal(got, want)
    # the TMA-staged kernel at full size (the plan's default for k >= 8), on
    # the level its stages fit best -- wide groups of 64 rows at k = 8, of 32
    # at k = 32, the 16-row groups at k = 128 -- bit for bit too
    staged = CsrPlan(ctx, a, PLAN_ROW_GROUPS)
    assert staged.properties() & PLAN_HAS_STAGED_SPMM
    assert staged.spmm_stage_rows(k) == {8: 64, 32: 32, 128: 16}[k]
    assert bits_equal(run_spmm(ctx, a, b_d, a_h.rows, a_h.cols, k, alpha, staged), want)
    del got, want
    ctx.set_determinism(Determinism.kBackendDefault)
    for plan in (None, CsrPlan(ctx, a), staged):
        got = run_spmm(ctx, a, b_d, a_h.rows, a_h.cols, k, alpha, plan)
        spmm_default_check(restatement, a_h, b, got, alpha,
                           lambda n, s: oracle.gamma(n + 2, np.float32) * s)
        if plan is not None:
            plan.close()
    assert ctx.device_status() == 0
    ctx.close()


@pytest.mark.parametrize("k", [8, 32, 128])
def test_block16_65536_spmm(cuda_lib, restatement, k):
    """The 16 x 16-block matrix through the tensor-core plan (3xTF32): within
    (n + 64) 2^-22 |alpha| sum|a b| of the FP64 oracle; DETERMINISTIC through
    the same plan bit for bit."""
    if "bk" not in _CACHE:
        _CACHE["bk"] = synthetic.block_sparse(65_536, 16, 0.02, seed=2, dtype=np.float32)
    a_h = _CACHE["bk"]
    assert a_h.rows == 65_536 and a_h.nnz == 85_983_232
    rng = np.random.default_rng(3)
    b = rng.standard_normal((a_h.cols, k), dtype=np.float32)
    alpha = 1.0
    ctx = context(Determinism.kBackendDefault)
    a = csr(a_h.rows, a_h.cols, a_h.ptr, a_h.idx, a_h.val)
    plan = CsrPlan(ctx, a)
    assert plan.properties() & PLAN_HAS_BLOCKS16
    b_d = dev(b)
    got = run_spmm(ctx, a, b_d, a_h.rows, a_h.cols, k, alpha, plan)
    spmm_default_check(restatement, a_h, b, got, alpha,
                       lambda n, s: (n + 64) * 2.0 ** -22 * s)
    assert ctx.device_status(clear=True) == 0
    ctx.set_determinism(Determinism.kDeterministic)
    got = run_spmm(ctx, a, b_d, a_h.rows, a_h.cols, k, alpha, plan)
    want = oracle.standard_spmm_rows(restatement, a_h.cols, a_h.ptr, a_h.idx, a_h.val, alpha, b,
                                     np.zeros((a_h.rows, k), np.float32))
    assert bits_equal(got, want)
    plan.close()
    ctx.close()


def _batch_views(g):
    mats, xs, ys = [], [], []
    for m in range(len(g["rows"])):
        n, z = int(g["rows"][m]), int(g["nnz"][m])
        pb, nb, rb = int(g["ptr_base"][m]), int(g["nz_base"][m]), int(g["row_base"][m])
        mats.append(CudaCsrArray(n, n, g["ptr"][pb:pb + n + 1], g["idx"][nb:nb + z],
                                 g["val"][nb:nb + z]))
        xs.append(CudaStridedVectorView(g["x"][rb:rb + n], n, writable=False))
        ys.append(CudaStridedVectorView(g["y"][rb:rb + n], n))
    return mats, xs, ys


def _check_batch(restatement, g, exact_mode, alpha, beta, y0):
    """Every matrix of the batch against the oracle (bit for bit, or within
    the bound), copying 256 matrices at a time to the host."""
    from concurrent.futures import ThreadPoolExecutor
    count = len(g["rows"])
    y_all = host(g["y"])
    worst = [0.0]

    def one(m, ptr, idx, val, x, y, y_init):
        if exact_mode:
            want = restatement.compat_spmv(ptr, idx, val, alpha, x, beta, y_init.copy())
            assert bits_equal(y, want), m
        else:
            exact, absval = restatement.extended(OP_NONE, len(ptr) - 1, len(x), ptr, idx, val, x)
            ref = alpha * exact + beta * y_init.astype(np.longdouble)
            rep = oracle.error_report(y, ref, absval, np.diff(ptr), np.float64, alpha,
                                      np.abs(beta * y_init))
            assert rep["max_ratio_to_bound"] <= 1.0, (m, rep)
            worst[0] = max(worst[0], rep["max_ratio_to_bound"])

    with ThreadPoolExecutor(max_workers=oracle._threads(None)) as ex:
        for m0 in range(0, count, 256):
            m1 = min(count, m0 + 256)
            p0, p1 = int(g["ptr_base"][m0]), int(g["ptr_base"][m1 - 1] + g["rows"][m1 - 1] + 1)
            z0 = int(g["nz_base"][m0])
            z1 = int(g["nz_base"][m1 - 1] + g["nnz"][m1 - 1])
            ptr = g["ptr"][p0:p1].cpu().numpy()
            idx = g["idx"][z0:z1].cpu().numpy()
            val = g["val"][z0:z1].cpu().numpy()
            xs = g["x"][int(g["row_base"][m0]):int(g["row_base"][m1 - 1] + g["rows"][m1 - 1])]
            xh = xs.cpu().numpy()
            futs = []
            for m in range(m0, m1):
                n = int(g["rows"][m])
                pb = int(g["ptr_base"][m]) - p0
                nb = int(g["nz_base"][m]) - z0
                rb = int(g["row_base"][m]) - int(g["row_base"][m0])
                z = int(g["nnz"][m])
                rg = int(g["row_base"][m])
                futs.append(ex.submit(one, m, ptr[pb:pb + n + 1], idx[nb:nb + z], val[nb:nb + z],
                                      xh[rb:rb + n], y_all[rg:rg + n], y0[rg:rg + n]))
            for f in futs:
                f.result()
    return worst[0]


def test_banded_batch_4096(cuda_lib, restatement):
    """All 4096 matrices (sum of rows ~33M, ~1.1e9 nonzeros) through one
    graph-captured persistent launch: bit for bit in DETERMINISTIC mode, within
    the bound in BACKEND_DEFAULT."""
    g = synthetic.banded_batch_device(4096)
    assert len(g["rows"]) == 4096
    mats, xs, ys = _batch_views(g)
    rng = np.random.default_rng(33)
    y0 = rng.uniform(-1, 1, int(g["rows"].sum()))
    alpha, beta = 1.0, 0.5
    ctx = context()
    batch = CudaBatch(ctx, mats, xs, ys)
    batch.capture(alpha, beta)
    g["y"].copy_(torch.from_numpy(y0))
    batch.spmv(alpha, beta)  # graph replay
    _check_batch(restatement, g, True, alpha, beta, y0)
    batch.close()
    ctx.set_determinism(Determinism.kBackendDefault)
    batch = CudaBatch(ctx, mats, xs, ys)
    batch.capture(alpha, beta)
    g["y"].copy_(torch.from_numpy(y0))
    batch.spmv(alpha, beta)
    _check_batch(restatement, g, False, alpha, beta, y0)
    batch.close()
    assert ctx.device_status() == 0
    ctx.close()
    del mats, xs, ys, g
    torch.cuda.empty_cache()
