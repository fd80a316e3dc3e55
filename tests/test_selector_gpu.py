"""GPU parity of the learned variant selector: the CUDA feature kernels and
the MLP forward / backward / Adam kernels against the float64 CPU oracle
(oracle/mlp_oracle.py), the exhaustive autotuner, plan-time selection, and --
on the timings the autotuner measured on B200 (tests/golden/
selector_timings.npz) -- what the trained network gains over the default
variant on the 400 held-out matrices."""

import ctypes
import os

import numpy as np
import pytest
import torch

from asc_cpp_b200 import selector, synthetic
from asc_cpp_b200._abi import Determinism, Variant
from asc_cpp_b200.sparse_cuda import CsrPlan, CudaCsrSpmv, CudaCsrSpmvWorkspaceSize
from oracle import mlp_oracle

from gpu_util import assert_within_bound, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _matrices():
    rng = np.random.default_rng(71)
    yield synthetic.banded(rng, 3000, 7), 8
    yield synthetic.random_csr(rng, 2000, 1500, 90, np.float32, 0.3), 4
    yield synthetic.laplacian_2d(60), 8
    yield synthetic.random_csr(rng, 500, 50000, 3, np.float64, 0.0), 8


def test_features_match_oracle(cuda_lib):
    ctx = context()
    for m, eb in _matrices():
        a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
        got = host(selector.matrix_features(ctx, a)).astype(np.float64)
        want = mlp_oracle.features(m.rows, m.cols, m.ptr, m.idx, eb)
        np.testing.assert_allclose(got, want, rtol=2e-7, atol=1e-7)
    ctx.close()


def test_forward_backward_adam_match_oracle(cuda_lib):
    ctx = context()
    rng = np.random.default_rng(5)
    v, b = 8, 37
    p = (rng.standard_normal(mlp_oracle.param_count(v)) * 0.3).astype(np.float32)
    x = rng.standard_normal((b, 12)).astype(np.float32)
    t = rng.standard_normal((b, v)).astype(np.float32)
    mlp = selector.Mlp(ctx, v, params=p)
    xd, td = dev(x), dev(t)
    grads, loss, y = mlp.gradient(xd, td)
    _, _, y_ref = mlp_oracle.forward(p.astype(np.float64), x, v)
    np.testing.assert_allclose(host(y), y_ref, rtol=1e-4, atol=1e-5)
    g_ref = mlp_oracle.backward(p.astype(np.float64), x, t, v)
    g = host(grads).astype(np.float64)
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-4 * scale
    np.testing.assert_allclose(host(loss).mean(), mlp_oracle.loss(p, x, t, v), rtol=1e-4)
    # one Adam step from zero moments
    m0 = np.zeros_like(p)
    params = torch.from_numpy(p.copy()).cuda()
    mm = torch.zeros_like(params)
    ss = torch.zeros_like(params)
    ctx.check(ctx._lib.asc_sb_selector_adam(ctx.handle, params.data_ptr(), grads.data_ptr(),
                                            mm.data_ptr(), ss.data_ptr(), params.numel(),
                                            ctypes.c_float(1e-2), ctypes.c_float(0.9),
                                            ctypes.c_float(0.999), ctypes.c_float(1e-8), 1))
    p_ref, _, _ = mlp_oracle.adam(p.astype(np.float64), g, m0, m0, 1e-2, 0.9, 0.999, 1e-8, 1)
    np.testing.assert_allclose(host(params), p_ref, rtol=1e-5, atol=1e-6)
    ctx.close()


def test_training_fits_a_teacher(cuda_lib):
    """The GPU training loop drives the loss down on targets of a random
    teacher network (a learnable problem with known optimum 0)."""
    ctx = context()
    rng = np.random.default_rng(9)
    v = 8
    teacher = (rng.standard_normal(mlp_oracle.param_count(v)) * 0.2)
    x = rng.standard_normal((512, 12)).astype(np.float32)
    t = mlp_oracle.forward(teacher, x, v)[2].astype(np.float32)
    mlp = selector.Mlp(ctx, v, seed=1)
    hist = mlp.train(dev(x), dev(t), epochs=1500, lr=3e-3)
    assert hist[-1] < 0.05 * hist[0]
    ctx.close()


def test_autotune_picks_the_fastest_and_plan_uses_it(cuda_lib, restatement):
    rng = np.random.default_rng(12)
    m = synthetic.power_law(200_000, seed=3, dtype=np.float64)
    ctx = context(Determinism.kBackendDefault)
    a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
    x_h = rng.uniform(-1, 1, m.cols)
    x = dev(x_h)
    y = dev(np.zeros(m.rows))
    plan = CsrPlan(ctx, a)
    variants = np.array([v for v, _ in selector.VARIANTS], np.int32)
    lanes = np.array([l for _, l in selector.VARIANTS], np.int32)
    ms = np.zeros(len(variants), np.float32)
    xd, yd = vec(x, writable=False).describe(), vec(y).describe()
    ctx.check(ctx._lib.asc_sb_plan_autotune(ctx.handle, plan.handle, ctypes.byref(xd),
                                            ctypes.byref(yd), len(variants), variants.ctypes.data,
                                            lanes.ctypes.data, 3, ms.ctypes.data))
    assert (ms > 0).all()
    got_v, got_l = ctypes.c_int32(), ctypes.c_int32()
    ctx.check(ctx._lib.asc_sb_plan_variant(plan.handle, ctypes.byref(got_v), ctypes.byref(got_l)))
    best = int(np.argmin(ms))
    assert (got_v.value, got_l.value) == (int(variants[best]), int(lanes[best]))
    # the plan's product runs the picked variant within the bound
    y0 = rng.uniform(-1, 1, m.rows)
    yt = dev(y0)
    plan.csr_spmv(1.25, vec(x, writable=False), 0.5, vec(yt))
    exact, absval = restatement.extended(0, m.rows, m.cols, m.ptr, m.idx, m.val, x_h)
    ref = 1.25 * exact + 0.5 * y0.astype(np.longdouble)
    assert_within_bound(host(yt), exact, absval, np.diff(m.ptr), np.float64, 1.25,
                        np.abs(0.5 * y0), ref)
    plan.close()
    ctx.close()


def test_installed_selector_picks_a_variant(cuda_lib, restatement):
    if not os.path.exists(selector.WEIGHTS):
        pytest.skip("no trained selector weights shipped")
    rng = np.random.default_rng(13)
    ctx = context(Determinism.kBackendDefault)
    selector.install(ctx)
    allowed = set(selector.VARIANTS)
    for m, _ in _matrices():
        m64 = m.astype(np.float64)
        a = csr(m64.rows, m64.cols, m64.ptr, m64.idx, m64.val)
        plan = CsrPlan(ctx, a)
        v, l = ctypes.c_int32(), ctypes.c_int32()
        ctx.check(ctx._lib.asc_sb_plan_variant(plan.handle, ctypes.byref(v), ctypes.byref(l)))
        assert (v.value, l.value) in allowed
        x_h = rng.uniform(-1, 1, m64.cols)
        y = dev(np.zeros(m64.rows))
        plan.csr_spmv(1.0, vec(dev(x_h), writable=False), 0.0, vec(y))
        exact, absval = restatement.extended(0, m64.rows, m64.cols, m64.ptr, m64.idx, m64.val,
                                             x_h)
        assert_within_bound(host(y), exact, absval, np.diff(m64.ptr), np.float64, 1.0,
                            np.zeros(m64.rows), exact)
        plan.close()
    # DETERMINISTIC contexts ignore the selector: plans record no variant
    ctx.set_determinism(Determinism.kDeterministic)
    m, _ = next(_matrices())
    plan = CsrPlan(ctx, csr(m.rows, m.cols, m.ptr, m.idx, m.val))
    v, l = ctypes.c_int32(), ctypes.c_int32()
    ctx.check(ctx._lib.asc_sb_plan_variant(plan.handle, ctypes.byref(v), ctypes.byref(l)))
    assert v.value == int(Variant.kAuto)
    plan.close()
    ctx.close()


def test_trained_selector_on_held_out_matrices(cuda_lib):
    """Trains the MLP with the library's kernels on the first 1600 matrices
    of the B200 autotune timings and scores its picks on the other 400:
    within 10% of exhaustive autotuning, and faster than the default
    variant."""
    path = os.path.join(GOLDEN, "selector_timings.npz")
    if not os.path.exists(path):
        pytest.skip("selector timings not collected")
    data = dict(np.load(path))
    ctx = context()
    _, report, history = selector.train_and_evaluate(ctx, data, 1600, epochs=3000)
    assert history[-1] < history[0]
    assert report["mean_slowdown_vs_exhaustive"] <= 1.10, report
    assert report["geomean_speedup_vs_default"] > 1.0, report
    ctx.close()
