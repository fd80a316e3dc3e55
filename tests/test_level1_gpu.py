"""GPU parity of Level-1 sparse BLAS on indexed vectors (asc_sb_standard_level1,
the replacement of internal_sparse_cuda::StandardLevel1Erased): dot (plain and
conjugated), axpy, gather, gather-zero and scatter against the reference's own
outputs (tests/golden/level1_cases.npz, made from the values of
tests/sparse/standard_blas_test.cc:69-173 and a seeded random case), the
contracted dot against its error bound, strided dense operands, and the
validation failures of operations.cc:1122-1212."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200._abi import Determinism, ErrorCode, IndexedDesc, Level1Op
from asc_cpp_b200.sparse_cuda import AscError, CudaLevel1, CudaStridedVectorView, _kind

from gpu_util import bits_equal, context, dev, gamma, host, vec

pytestmark = pytest.mark.gpu

TAGS = {"f64": np.float64, "f32": np.float32, "z": np.complex128, "c": np.complex64}


def _alpha(dt):
    return (0.75 - 1.5j) if np.iscomplexobj(dt(0)) else 2.0


@pytest.mark.parametrize("tag", list(TAGS))
def test_level1_matches_reference_bit_for_bit(cuda_lib, level1_cases, tag):
    g = level1_cases
    ctx = context()
    for name in ("ka", "rand"):
        idx, val, x = g[f"{name}_idx_{tag}"], g[f"{name}_val_{tag}"], g[f"{name}_x_{tag}"]
        for op in range(5):
            for conj in ((0, 1) if op == 0 else (0,)):
                key = f"{name}_op{op}_conj{conj}_{tag}"
                v_d, x_d = dev(val), dev(x)
                r_d = torch.zeros(1, dtype=v_d.dtype, device="cuda")
                CudaLevel1(ctx, op, dev(idx), v_d, vec(x_d), r_d, _alpha(TAGS[tag]), bool(conj))
                assert bits_equal(host(v_d), g[key + "_val"]), key
                assert bits_equal(host(x_d), g[key + "_x"]), key
                if op == Level1Op.kDot:
                    assert bits_equal(host(r_d), g[key + "_res"]), key
    ctx.close()


@pytest.mark.parametrize("tag", list(TAGS))
def test_large_deterministic_dot_and_elementwise(cuda_lib, restatement, tag):
    """300k stored entries over a 2M dense vector: the stored-order dot and
    every element-wise operation stay bit-identical to the oracle."""
    dt = TAGS[tag]
    rng = np.random.default_rng(17)
    n, nnz = 2_000_000, 300_000
    idx = np.sort(rng.choice(n, nnz, replace=False)).astype(np.int64)
    cplx = np.iscomplexobj(dt(0))
    val = (rng.uniform(-1, 1, nnz) + (1j * rng.uniform(-1, 1, nnz) if cplx else 0)).astype(dt)
    x = (rng.uniform(-1, 1, n) + (1j * rng.uniform(-1, 1, n) if cplx else 0)).astype(dt)
    ctx = context()
    idx_d = dev(idx)
    for op in range(5):
        for conj in ((0, 1) if op == 0 else (0,)):
            v_want, x_want, r_want = restatement.level1(op, conj, idx, val, _alpha(dt), x)
            v_d, x_d = dev(val), dev(x)
            r_d = torch.zeros(1, dtype=v_d.dtype, device="cuda")
            CudaLevel1(ctx, op, idx_d, v_d, vec(x_d), r_d, _alpha(dt), bool(conj))
            assert bits_equal(host(v_d), v_want) and bits_equal(host(x_d), x_want), (op, conj)
            if op == Level1Op.kDot:
                assert bits_equal(host(r_d), np.array([r_want], dt)), (op, conj)
    ctx.close()


@pytest.mark.parametrize("tag", list(TAGS))
def test_contracted_dot_within_bound_and_reproducible(cuda_lib, tag):
    """BACKEND_DEFAULT dot (grid reduction with a fixed tree): within
    gamma_{n+2} * sum |v_k| |x_{i_k}| (doubled for complex products) of the
    long-double sum, and the same bits on every run."""
    dt = TAGS[tag]
    rng = np.random.default_rng(23)
    n, nnz = 3_000_000, 1_000_000
    idx = np.sort(rng.choice(n, nnz, replace=False)).astype(np.int64)
    cplx = np.iscomplexobj(dt(0))
    val = (rng.uniform(-1, 1, nnz) + (1j * rng.uniform(-1, 1, nnz) if cplx else 0)).astype(dt)
    x = (rng.uniform(-1, 1, n) + (1j * rng.uniform(-1, 1, n) if cplx else 0)).astype(dt)
    ctx = context(Determinism.kBackendDefault)
    idx_d, v_d, x_d = dev(idx), dev(val), dev(x)
    real_t = np.float32 if dt in (np.float32, np.complex64) else np.float64
    for conj in (0, 1):
        results = []
        for _ in range(3):
            r_d = torch.zeros(1, dtype=v_d.dtype, device="cuda")
            CudaLevel1(ctx, Level1Op.kDot, idx_d, v_d, vec(x_d, writable=False), r_d,
                       conjugated=bool(conj))
            results.append(host(r_d))
        assert all(bits_equal(r, results[0]) for r in results[1:])
        xv = x[idx]
        vv = np.conj(val) if conj else val
        if cplx:
            re = (vv.real.astype(np.longdouble) * xv.real - vv.imag.astype(np.longdouble) * xv.imag)
            im = (vv.real.astype(np.longdouble) * xv.imag + vv.imag.astype(np.longdouble) * xv.real)
            exact = complex(float(re.sum()), float(im.sum()))
            mag = float((np.abs(val).astype(np.longdouble) * np.abs(xv)).sum()) * 2
        else:
            exact = float((vv.astype(np.longdouble) * xv).sum())
            mag = float((np.abs(vv).astype(np.longdouble) * np.abs(xv)).sum())
        bound = gamma(np.array([nnz + 2]), real_t)[0] * mag
        assert abs(complex(results[0][0]) - exact) <= bound, (results[0][0], exact, bound)
    ctx.close()


def test_strided_dense_operand(cuda_lib, restatement):
    """Dense x with stride 3 and offset 2: only the addressed slots change."""
    rng = np.random.default_rng(29)
    ext, nnz = 5000, 1200
    idx = np.sort(rng.choice(ext, nnz, replace=False)).astype(np.int64)
    val = rng.uniform(-1, 1, nnz)
    full = rng.uniform(-1, 1, 2 + 3 * ext)
    ctx = context()
    for op in (Level1Op.kDot, Level1Op.kAxpy, Level1Op.kGather, Level1Op.kGatherZero,
               Level1Op.kScatter):
        x = full[2::3].copy()
        v_want, x_want, r_want = restatement.level1(int(op), 0, idx, val, -0.5, x)
        f_d, v_d = dev(full), dev(val)
        r_d = torch.zeros(1, dtype=torch.float64, device="cuda")
        CudaLevel1(ctx, op, dev(idx), v_d, vec(f_d, extent=ext, stride=3, offset=2), r_d, -0.5)
        f_got = host(f_d)
        assert bits_equal(f_got[2::3].copy(), x_want)
        untouched = np.ones(full.size, bool)
        untouched[2::3] = False
        assert bits_equal(f_got[untouched], full[untouched])
        assert bits_equal(host(v_d), v_want)
        if op == Level1Op.kDot:
            assert host(r_d)[0] == r_want
    ctx.close()


def test_empty_and_zero_alpha(cuda_lib):
    ctx = context()
    x_d = dev(np.arange(6, dtype=np.float64))
    empty_i = torch.zeros(0, dtype=torch.int64, device="cuda")
    empty_v = torch.zeros(0, dtype=torch.float64, device="cuda")
    r_d = dev(np.array([7.0]))
    CudaLevel1(ctx, Level1Op.kDot, empty_i, empty_v, vec(x_d), r_d)
    assert host(r_d)[0] == 0.0
    for op in (Level1Op.kAxpy, Level1Op.kGather, Level1Op.kGatherZero, Level1Op.kScatter):
        CudaLevel1(ctx, op, empty_i, empty_v, vec(x_d), alpha=3.0)
    idx = dev(np.array([1, 4], np.int64))
    v = dev(np.array([np.nan, 2.0]))
    CudaLevel1(ctx, Level1Op.kAxpy, idx, v, vec(x_d), alpha=0.0)  # alpha 0: nothing touched
    assert host(x_d).tolist() == [0.0, 1.0, 2.0, 3.0, 4.0, 5.0]
    ctx.close()


def _raw(ctx, op, idx_t, val_t, dense, result=None, *, extent=None, trusted=1,
         sparse_writable=None, dense_writable=None, result_extent=1):
    d = IndexedDesc()
    d.indices = idx_t.data_ptr() if idx_t.numel() else None
    d.values = val_t.data_ptr() if val_t.numel() else None
    d.memory_space = 2
    d.element_kind = _kind(val_t.dtype)
    d.nonzeros = val_t.numel()
    d.dense_extent = dense.extent if extent is None else extent
    d.writable = 1 if sparse_writable is None else sparse_writable
    d.canonical_structure_trusted = trusted
    dd = dense.describe()
    # a descriptor's mutability must equal what the operation needs
    dd.writable = int(op in (Level1Op.kAxpy, Level1Op.kGatherZero, Level1Op.kScatter))
    if dense_writable is not None:
        dd.writable = dense_writable
    rd = CudaStridedVectorView(result, result_extent).describe() if result is not None else None
    return ctx._lib.asc_sb_standard_level1(ctx.handle, int(op), 0, 1.0, 0.0, ctypes.byref(d),
                                           ctypes.byref(dd),
                                           ctypes.byref(rd) if rd is not None else None)


def test_validation_failures(cuda_lib):
    """The reference's rejections: extents that disagree, a result that is not
    one element or overlaps an input, operands that overlap, untrusted
    structure, read-only outputs, unknown operation or conjugation."""
    ctx = context()
    idx = dev(np.array([0, 3], np.int64))
    val = dev(np.array([1.0, 2.0]))
    x = dev(np.zeros(5))
    r = dev(np.zeros(2))
    dense = vec(x)
    assert _raw(ctx, Level1Op.kDot, idx, val, dense, r, extent=4) == ErrorCode.kShape
    assert _raw(ctx, Level1Op.kDot, idx, val, dense, r, result_extent=2) == ErrorCode.kShape
    assert _raw(ctx, Level1Op.kDot, idx, val, dense, None) == ErrorCode.kInvalidArgument
    assert _raw(ctx, Level1Op.kDot, idx, val, dense, r, trusted=0) == ErrorCode.kInvalidArgument
    assert (_raw(ctx, Level1Op.kGather, idx, val, dense, sparse_writable=0)
            == ErrorCode.kInvalidArgument)
    assert (_raw(ctx, Level1Op.kScatter, idx, val, dense, dense_writable=0)
            == ErrorCode.kInvalidArgument)
    assert (_raw(ctx, Level1Op.kDot, idx, val, dense, r, dense_writable=1)
            == ErrorCode.kInvalidArgument)
    # values that alias the dense vector
    big = dev(np.zeros(8))
    alias_v = big[:2]
    alias_x = CudaStridedVectorView(big, 5, 1, 1, True)
    assert _raw(ctx, Level1Op.kAxpy, idx, alias_v, alias_x) == ErrorCode.kInvalidArgument
    # a dot result inside the dense vector
    assert (_raw(ctx, Level1Op.kDot, idx, val, vec(big, extent=5), big[4:5])
            == ErrorCode.kInvalidArgument)
    # nonzeros above the dense extent
    assert _raw(ctx, Level1Op.kDot, dev(np.arange(3, dtype=np.int64)), dev(np.ones(3)),
                vec(dev(np.zeros(2))), r[:1]) == ErrorCode.kShape
    assert (ctx._lib.asc_sb_standard_level1(ctx.handle, 9, 0, 1.0, 0.0, None, None, None)
            == ErrorCode.kInvalidArgument)
    assert (ctx._lib.asc_sb_standard_level1(ctx.handle, 0, 5, 1.0, 0.0, None, None, None)
            == ErrorCode.kInvalidArgument)
    with pytest.raises(AscError) as e:  # a result of another element kind
        CudaLevel1(ctx, Level1Op.kDot, idx, val, vec(x), torch.zeros(1, device="cuda"))
    assert e.value.code == ErrorCode.kInvalidArgument
    ctx.close()
