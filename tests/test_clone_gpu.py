"""GPU checks of the host -> device clones (asc_sb_clone_csr /
asc_sb_clone_indexed, the copy half of internal_sparse_cuda::CloneCsrErased
and CloneIndexedErased, src/sparse/cuda/operations.cc:696-880): the device
arrays equal the host arrays byte for byte for pageable sources small and
large (the staged path, several 16 MiB chunks), page-locked sources (direct
DMA) and every element kind; a pageable source may change once the call has
returned; and the validation failures of the reference leave the
destination untouched."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200 import synthetic
from asc_cpp_b200._abi import ErrorCode, FormatKind, IndexedDesc, MemorySpace, SparseDesc
from asc_cpp_b200.sparse_cuda import (AscError, CudaCloneCsr, CudaCloneIndexedVector,
                                      _host_sparse_desc)

from gpu_util import bits_equal, context, host

pytestmark = pytest.mark.gpu


def _same(dev_t, host_a):
    return bits_equal(host(dev_t), np.asarray(host_a))


@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.complex64])
def test_clone_csr_pageable_small_and_large(cuda_lib, dt):
    ctx = context()
    rng = np.random.default_rng(3)
    small = synthetic.random_csr(rng, 300, 200, 20, np.float64, 0.1)
    big = synthetic.power_law(1_500_000, 12.0, 1.2, 4096, seed=4)  # ~18M entries: staged
    for m in (small, big):
        val = m.val.astype(dt) if not np.iscomplexobj(dt(0)) else \
            (m.val + 1j * m.val[::-1]).astype(dt)
        a = CudaCloneCsr(ctx, m.rows, m.cols, m.ptr, m.idx, val)
        assert _same(a.offsets, m.ptr) and _same(a.indices, m.idx) and _same(a.values, val)
    ctx.close()


def test_clone_csr_pinned_source_and_reuse_after_return(cuda_lib):
    ctx = context()
    m = synthetic.power_law(1_000_000, 10.0, 1.0, 2048, seed=5)
    ptr = torch.from_numpy(m.ptr).pin_memory()
    idx = torch.from_numpy(m.idx).pin_memory()
    val = torch.from_numpy(m.val).pin_memory()
    a = CudaCloneCsr(ctx, m.rows, m.cols, ptr, idx, val)
    torch.cuda.synchronize()
    assert _same(a.offsets, m.ptr) and _same(a.indices, m.idx) and _same(a.values, m.val)
    # a pageable source is fully read when the call returns
    src_val = m.val.copy()
    b = CudaCloneCsr(ctx, m.rows, m.cols, m.ptr, m.idx, src_val)
    src_val[:] = -7.0
    assert _same(b.values, m.val)
    ctx.close()


def test_clone_indexed(cuda_lib):
    ctx = context()
    rng = np.random.default_rng(8)
    for n, nnz in ((1000, 17), (40_000_000, 3_000_000)):
        idx = np.sort(rng.choice(n, nnz, replace=False)).astype(np.int64)
        val = rng.standard_normal(nnz) + 1j * rng.standard_normal(nnz)
        d_idx, d_val = CudaCloneIndexedVector(ctx, idx, val, n)
        assert _same(d_idx, idx) and _same(d_val, val)
    ctx.close()


def test_clone_empty(cuda_lib):
    ctx = context()
    a = CudaCloneCsr(ctx, 5, 4, np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0))
    assert _same(a.offsets, np.zeros(6, np.int64)) and a.nnz == 0
    d_idx, d_val = CudaCloneIndexedVector(ctx, np.zeros(0, np.int64), np.zeros(0), 10)
    assert d_idx.numel() == 0
    ctx.close()


def test_clone_validation(cuda_lib):
    """operations.cc:696-721, 802-831: host CSR source only, matching device
    destination, trusted structure, no overlap; nothing is written."""
    ctx = context()
    m = synthetic.random_csr(np.random.default_rng(9), 50, 40, 6, np.float64)
    dev = torch.device("cuda", 0)
    off = torch.full((51,), -1, dtype=torch.int64, device=dev)
    idx = torch.full((m.nnz,), -1, dtype=torch.int64, device=dev)
    val = torch.full((m.nnz,), -1.0, dtype=torch.float64, device=dev)

    def dst(rows=50, cols=40, fmt=FormatKind.kCsr, space=MemorySpace.kDevice, values=val):
        d = SparseDesc()
        d.structure_first, d.structure_second = off.data_ptr(), idx.data_ptr()
        d.values = values.data_ptr()
        d.memory_space, d.element_kind = int(space), 1
        d.format, d.canonical_structure_trusted = int(fmt), 1
        d.rows, d.columns, d.nonzeros = rows, cols, m.nnz
        return d

    def call(src, d):
        return ctx._lib.asc_sb_clone_csr(ctx.handle, ctypes.byref(src), ctypes.byref(d))

    src = _host_sparse_desc(50, 40, m.ptr, m.idx, m.val, FormatKind.kCsr)
    csc = _host_sparse_desc(50, 40, m.ptr, m.idx, m.val, FormatKind.kCsc)
    assert call(csc, dst()) == ErrorCode.kMemoryAccess
    on_device = _host_sparse_desc(50, 40, m.ptr, m.idx, m.val, FormatKind.kCsr)
    on_device.memory_space = int(MemorySpace.kDevice)
    assert call(on_device, dst()) == ErrorCode.kMemoryAccess
    untrusted = _host_sparse_desc(50, 40, m.ptr, m.idx, m.val, FormatKind.kCsr)
    untrusted.canonical_structure_trusted = 0
    assert call(untrusted, dst()) == ErrorCode.kInvalidArgument
    assert call(src, dst(rows=49)) == ErrorCode.kShape
    assert call(src, dst(space=MemorySpace.kHost)) == ErrorCode.kMemoryAccess
    f32 = torch.zeros(m.nnz, dtype=torch.float32, device=dev)
    d = dst(values=f32)
    d.element_kind = 0
    assert call(src, d) == ErrorCode.kShape
    alias = dst()
    alias.values = idx.data_ptr()  # values over the index array
    assert call(src, alias) == ErrorCode.kInvalidArgument
    torch.cuda.synchronize()
    assert (off.cpu() == -1).all() and (idx.cpu() == -1).all() and (val.cpu() == -1).all()
    s_idx, s_val = IndexedDesc(), IndexedDesc()
    s_idx.memory_space = int(MemorySpace.kDevice)
    assert ctx._lib.asc_sb_clone_indexed(ctx.handle, ctypes.byref(s_idx),
                                         ctypes.byref(s_val)) == ErrorCode.kMemoryAccess
    with pytest.raises(AscError):
        CudaCloneIndexedVector(ctx, np.array([0, 1, 2], np.int64), np.ones(3), 2)
    ctx.close()
