"""GPU checks of the pointwise evaluation entry point (asc_sb_evaluate, the
replacement of internal_sparse_cuda::EvaluateErased,
src/sparse/cuda/operations.cc:1051-1120): copy, negate, add, subtract and
multiply over one sparsity structure with view and scalar operands, compressed
and coordinate (rank 3) storage, FP32 and FP64, against numpy on the same
values (one rounding per element, as the reference kernel does), and the
reference's validation failures, which leave the destination untouched."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200._abi import ErrorCode, OperandDesc, TensorDesc

from gpu_util import bits_equal, context, dev, host

pytestmark = pytest.mark.gpu

COPY, NEGATE, ADD, SUBTRACT, MULTIPLY = range(5)
VIEW, SCALAR = 0, 1
COORDINATE, CSR = 0, 1
DEVICE = 2


class Tensor:
    """A device sparse tensor's structure arrays and extents (kept alive)."""

    def __init__(self, first, second, fmt, extents):
        self.first, self.second = first, second
        self.extents = (ctypes.c_int64 * len(extents))(*extents)
        self.fmt = fmt
        self.rank = len(extents)

    def desc(self, values):
        d = TensorDesc()
        d.structure_first = self.first.data_ptr() if self.first is not None else None
        d.structure_second = self.second.data_ptr() if self.second is not None else None
        d.values = values.data_ptr() if values.numel() else None
        d.memory_space = DEVICE
        d.element_kind = 0 if values.dtype == torch.float32 else 1
        d.format = self.fmt
        d.canonical_structure_trusted = 1
        d.rank = self.rank
        d.extents = ctypes.cast(self.extents, ctypes.POINTER(ctypes.c_int64))
        d.nonzeros = values.numel()
        return d


def view(t, values):
    o = OperandDesc()
    o.kind = VIEW
    o.view = t.desc(values)
    return o


def scalar(t, value, like):
    """A scalar operand; its element kind is that of the tensor `like`."""
    o = OperandDesc()
    o.kind = SCALAR
    o.view = t.desc(like)
    o.scalar = value
    return o


def evaluate(ctx, op, left, right, dest):
    return ctx._lib.asc_sb_evaluate(ctx.handle, op, ctypes.byref(left),
                                    ctypes.byref(right) if right is not None else None,
                                    ctypes.byref(dest))


def structures(rng, nnz):
    # a 40 x 50 CSR structure and a 6 x 7 x 8 coordinate one, nnz entries each
    # (evaluation never reads the structure's contents)
    ptr = dev(np.linspace(0, nnz, 41).astype(np.int64))
    idx = dev(rng.integers(0, 50, nnz).astype(np.int64))
    yield Tensor(ptr, idx, CSR, (40, 50))
    coords = dev(rng.integers(0, 6, (nnz, 3)).astype(np.int64))
    yield Tensor(coords, None, COORDINATE, (6, 7, 8))


@pytest.mark.parametrize("dt", [np.float32, np.float64], ids=["f32", "f64"])
def test_every_operation_and_operand_kind(cuda_lib, dt):
    rng = np.random.default_rng(4)
    ctx = context()
    nnz = 300
    a_h = rng.standard_normal(nnz).astype(dt)
    b_h = rng.standard_normal(nnz).astype(dt)
    for t in structures(rng, nnz):
        a, b = dev(a_h), dev(b_h)
        out = dev(np.zeros(nnz, dt))
        d = t.desc(out)
        cases = [(COPY, view(t, a), None, a_h.copy()),
                 (NEGATE, view(t, a), None, -a_h),
                 (ADD, view(t, a), view(t, b), a_h + b_h),
                 (SUBTRACT, view(t, a), view(t, b), a_h - b_h),
                 (MULTIPLY, view(t, a), view(t, b), a_h * b_h),
                 (MULTIPLY, view(t, a), scalar(t, 2.5, out), a_h * dt(2.5)),
                 (SUBTRACT, scalar(t, 1.0 / 3.0, out), view(t, b), dt(1.0 / 3.0) - b_h),
                 (COPY, scalar(t, -7.0, out), None, np.full(nnz, -7.0, dt))]
        for op, left, right, want in cases:
            assert evaluate(ctx, op, left, right, d) == 0, \
                ctx._lib.asc_sb_context_last_error(ctx.handle)
            assert bits_equal(host(out), want.astype(dt)), op
        # in place: the destination's own values as an operand
        out.copy_(a)
        assert evaluate(ctx, ADD, view(t, out), view(t, b), d) == 0
        assert bits_equal(host(out), a_h + b_h)
    ctx.close()


def test_validation_failures_leave_destination(cuda_lib):
    rng = np.random.default_rng(5)
    ctx = context()
    nnz = 64
    t, _ = list(structures(rng, nnz))
    a = dev(rng.standard_normal(nnz))
    out = dev(np.full(nnz, 9.0))
    d = t.desc(out)
    # another structure (a different index array) -> kInvalidArgument
    other = Tensor(t.first, dev(rng.integers(0, 50, nnz).astype(np.int64)), CSR, (40, 50))
    assert evaluate(ctx, COPY, view(other, a), None, d) == ErrorCode.kInvalidArgument
    assert b"identical structure" in ctx._lib.asc_sb_context_last_error(ctx.handle)
    # the same arrays with another shape -> kShape
    wide = Tensor(t.first, t.second, CSR, (40, 51))
    assert evaluate(ctx, COPY, view(wide, a), None, d) == ErrorCode.kShape
    # a view whose values partly overlap the destination's -> kInvalidArgument
    sd = view(t, out)
    sd.view.values = out.data_ptr() + 8
    assert evaluate(ctx, COPY, sd, None, d) == ErrorCode.kInvalidArgument
    # a scalar of another element kind, an unknown operation, a host destination
    s = scalar(t, 1.0, out)
    s.view.element_kind = 0
    assert evaluate(ctx, COPY, s, None, d) == ErrorCode.kInvalidArgument
    assert evaluate(ctx, 9, view(t, a), None, d) == ErrorCode.kInvalidArgument
    hd = t.desc(out)
    hd.memory_space = 0
    assert evaluate(ctx, COPY, view(t, a), None, hd) == ErrorCode.kMemoryAccess
    assert bits_equal(host(out), np.full(nnz, 9.0))
    # nothing stored: succeeds without a launch
    assert evaluate(ctx, NEGATE, view(t, out[:0]), None, t.desc(out[:0])) == 0
    ctx.close()
