"""GPU parity of the batched SpMV (one persistent work-queue launch for many
independent CSR matrices): DETERMINISTIC results equal the oracle bit for bit
for every matrix, through the direct launch, the per-matrix baseline, a CUDA
graph replay and every schedule; BACKEND_DEFAULT stays within the bound."""

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import Determinism, ErrorCode
from asc_cpp_b200.sparse_cuda import AscError, CudaBatch, CudaCsrArray

from gpu_util import assert_within_bound, bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu


def make_batch(dt, seed, count=40, misalign=None):
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        n = int(rng.integers(1, 3000))
        mats.append(synthetic.banded(rng, n, int(rng.integers(1, 32)), dtype=dt))
    mats.append(synthetic.Csr(0, 0, np.zeros(1, np.int64), np.zeros(0, np.int64),
                              np.zeros(0, dt)))
    mats.append(synthetic.random_csr(rng, 2500, 1700, 400, dt, 0.2))  # long rows
    xs = [rng.uniform(-1, 1, m.cols).astype(dt) for m in mats]
    ys = [rng.uniform(-1, 1, m.rows).astype(dt) for m in mats]
    dev_mats = []
    for i, m in enumerate(mats):
        if misalign is not None and i == misalign and m.nnz:
            # index array starting 8 bytes past a 16-byte boundary
            backing = dev(np.concatenate([np.zeros(1, np.int64), m.idx]))
            a = CudaCsrArray(m.rows, m.cols, dev(m.ptr), backing[1:], dev(m.val))
        else:
            a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
        dev_mats.append(a)
    return mats, xs, ys, dev_mats


def expected(restatement, mats, xs, ys, alpha, beta):
    out = []
    for m, x, y in zip(mats, xs, ys):
        e = y.copy()
        if m.rows:
            restatement.compat_spmv(m.ptr, m.idx, m.val, alpha, x, beta, e)
        out.append(e)
    return out


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("misalign", [None, 3])
def test_batch_bit_exact_every_path(cuda_lib, restatement, dt, misalign):
    mats, xs, ys, dmats = make_batch(dt, 7, misalign=misalign)
    want = expected(restatement, mats, xs, ys, 1.5, 0.5)
    ctx = context()
    xd = [dev(x) for x in xs]
    yd = [dev(y) for y in ys]
    batch = CudaBatch(ctx, dmats, [vec(x, writable=False) for x in xd], [vec(y) for y in yd])

    def run(fn):
        for t, y in zip(yd, ys):
            t.copy_(torch.from_numpy(y))
        fn()
        for i, (t, w) in enumerate(zip(yd, want)):
            assert bits_equal(host(t), w), i

    run(lambda: batch.spmv(1.5, 0.5))
    run(lambda: batch.spmv_per_matrix(1.5, 0.5))
    for chunk, ctas in ((1, 2), (32, 0), (7, 1)):
        batch.set_schedule(chunk, ctas)
        assert batch.schedule() == (chunk, ctas)
        run(lambda: batch.spmv(1.5, 0.5))
    batch.capture(1.5, 0.5)
    run(lambda: batch.spmv(1.5, 0.5))  # graph replay
    run(lambda: batch.spmv(1.5, 0.5))
    batch.close()
    ctx.close()


def test_batch_default_mode_within_bound(cuda_lib, restatement):
    mats, xs, ys, dmats = make_batch(np.float64, 11)
    ctx = context(Determinism.kBackendDefault)
    xd = [dev(x) for x in xs]
    yd = [dev(y) for y in ys]
    batch = CudaBatch(ctx, dmats, [vec(x, writable=False) for x in xd], [vec(y) for y in yd])
    batch.spmv(-2.0, 0.25)
    for m, x, y0, t in zip(mats, xs, ys, yd):
        if not m.rows:
            continue
        exact, absval = restatement.extended(0, m.rows, m.cols, m.ptr, m.idx, m.val, x)
        counts = np.diff(m.ptr)
        ref = -2.0 * exact + 0.25 * y0.astype(np.longdouble)
        assert_within_bound(host(t), exact, absval, counts, np.float64, -2.0,
                            np.abs(0.25 * y0), ref)
    batch.close()
    ctx.close()


def test_batch_autotune_keeps_results_exact(cuda_lib, restatement):
    mats, xs, ys, dmats = make_batch(np.float64, 13, count=60)
    ctx = context()
    xd = [dev(x) for x in xs]
    yd = [dev(y) for y in ys]
    batch = CudaBatch(ctx, dmats, [vec(x, writable=False) for x in xd], [vec(y) for y in yd])
    best = batch.autotune(1.0, 0.0, reps=2)
    assert best > 0
    chunk, ctas = batch.schedule()
    assert chunk >= 1 and ctas >= 0
    want = expected(restatement, mats, xs, ys, 1.0, 0.0)
    batch.spmv(1.0, 0.0)
    for t, w in zip(yd, want):
        assert bits_equal(host(t), w)
    batch.close()
    ctx.close()


def test_batch_rejects_overlapping_outputs(cuda_lib):
    rng = np.random.default_rng(3)
    m = synthetic.banded(rng, 100, 3)
    ctx = context()
    a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
    x = dev(rng.uniform(-1, 1, 100))
    shared = dev(np.zeros(150))
    with pytest.raises(AscError) as e:
        CudaBatch(ctx, [a, a], [vec(x, writable=False)] * 2,
                  [vec(shared[:100]), vec(shared[50:])])
    assert e.value.code == ErrorCode.kInvalidArgument
    # an output over another product's input
    with pytest.raises(AscError) as e:
        CudaBatch(ctx, [a, a], [vec(x, writable=False), vec(shared[:100], writable=False)],
                  [vec(shared[50:150]), vec(dev(np.zeros(100)))])
    assert e.value.code == ErrorCode.kInvalidArgument
    ctx.close()
