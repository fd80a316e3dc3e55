"""Failure paths on the GPU that fault, trap or hang nothing:

* allocation failures injected on the host, through a context allocator
  (asc_sb_context_set_allocator) that refuses a chosen request -- like the
  reference's TrackingDeviceResource::FailOnCall
  (tests/sparse_cuda/sparse_cuda_test.cc:40-85), for the memory the library
  allocates for itself: the growing scratch of triangular solves without a
  plan, the clone staging buffers and the selector's parameters.  The call
  reports ASC_SB_ALLOCATION, its outputs are untouched, the context goes on
  working, and every block handed out is given back;
* a dependency wait that runs out: the triangular solve's wait limit set to
  1 ns on a chain-shaped matrix, so its waits give up; the status word
  reports it, the launch ends, and the same context then solves correctly."""

import ctypes

import numpy as np
import pytest
import torch

from asc_cpp_b200 import selector, synthetic
from asc_cpp_b200._abi import ErrorCode, SparseBlasDiagonal, SparseBlasTranspose, SparseBlasTriangle
from asc_cpp_b200.sparse_cuda import AscError, CudaCloneCsr, CudaSparseTriangularSolve
from oracle import OP_NONE

from gpu_util import bits_equal, context, csr, dev, host, vec

pytestmark = pytest.mark.gpu

ALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32)
RELEASE = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                           ctypes.c_int32)
DEVICE, PINNED = 2, 1  # ASC_SB_DEVICE, ASC_SB_PINNED_HOST


class TrackingAllocator:
    """Serves the context's own requests from torch's allocators (as a host
    application that owns all memory would), counts them, and refuses the
    request numbered `fail_on` (0-based)."""

    def __init__(self, fail_on=None):
        self.fail_on = fail_on
        self.attempts = 0
        self.live = {}
        self._alloc = ALLOC(self._allocate)
        self._release = RELEASE(self._free)

    def _allocate(self, user, nbytes, space):
        call = self.attempts
        self.attempts += 1
        if call == self.fail_on:
            return None
        if space == DEVICE:
            t = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        else:
            t = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        self.live[t.data_ptr()] = t
        return t.data_ptr()

    def _free(self, user, pointer, nbytes, space):
        self.live.pop(pointer, None)

    def install(self, ctx):
        ctx.check(ctx._lib.asc_sb_context_set_allocator(
            ctx.handle, ctypes.cast(self._alloc, ctypes.c_void_p),
            ctypes.cast(self._release, ctypes.c_void_p), None))


def _chain(n):
    """Lower bidiagonal n x n matrix (each row depends on the one before)."""
    ptr = np.zeros(n + 1, np.int64)
    ptr[1] = 1
    ptr[2:] = 1 + 2 * np.arange(1, n, dtype=np.int64)
    idx = np.empty(int(ptr[-1]), np.int64)
    idx[0] = 0
    r = np.arange(1, n, dtype=np.int64)
    idx[1::2] = r - 1
    idx[2::2] = r
    rng = np.random.default_rng(5)
    val = rng.uniform(0.1, 0.5, idx.size)
    val[0] = 2.0
    val[2::2] = rng.uniform(1.5, 2.5, n - 1)
    return synthetic.Csr(n, n, ptr, idx, val)


def test_solve_scratch_allocation_failure(cuda_lib, restatement):
    m = _chain(50_000)
    rng = np.random.default_rng(6)
    b0 = rng.uniform(-1, 1, m.rows)
    ctx = context()
    alloc = TrackingAllocator(fail_on=0)
    alloc.install(ctx)
    a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
    b = dev(b0)
    with pytest.raises(AscError) as err:
        CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 1.0, a,
                                  SparseBlasTriangle.kLower, SparseBlasDiagonal.kNonUnit, vec(b))
    assert err.value.code == ErrorCode.kAllocation
    assert bits_equal(host(b), b0)  # untouched
    assert alloc.attempts == 1 and not alloc.live
    # the next request is served: the same context solves, bit for bit
    CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kLower,
                              SparseBlasDiagonal.kNonUnit, vec(b))
    want = restatement.triangular_solve(OP_NONE, 1, 0, m.rows, m.ptr, m.idx, m.val, 1.0,
                                        b0.reshape(-1, 1).copy(), 1, None, 1)
    assert bits_equal(host(b), want.reshape(-1))
    assert alloc.attempts == 2 and len(alloc.live) == 1
    assert ctx.device_status() == 0
    ctx.close()
    assert not alloc.live  # given back when the context went


def test_clone_staging_allocation_failure(cuda_lib):
    m = synthetic.power_law(600_000, 8.0, 1.0, 1024, seed=8)  # pageable arrays > 1 MiB: staged
    ctx = context()
    alloc = TrackingAllocator(fail_on=1)  # the second pinned staging buffer
    alloc.install(ctx)
    with pytest.raises(AscError) as err:
        CudaCloneCsr(ctx, m.rows, m.cols, m.ptr, m.idx, m.val)
    assert err.value.code == ErrorCode.kAllocation
    assert alloc.attempts == 2 and not alloc.live  # the first buffer was given back
    a = CudaCloneCsr(ctx, m.rows, m.cols, m.ptr, m.idx, m.val)
    assert bits_equal(host(a.indices), m.idx) and bits_equal(host(a.values), m.val)
    assert len(alloc.live) == 2
    ctx.close()
    assert not alloc.live


def test_selector_install_allocation_failure_keeps_previous(cuda_lib):
    ctx = context()
    selector.install(ctx)  # default allocator
    alloc = TrackingAllocator(fail_on=0)
    alloc.install(ctx)
    with pytest.raises(AscError) as err:
        selector.install(ctx)
    assert err.value.code == ErrorCode.kAllocation
    selector.install(ctx)  # served now; the first parameters go back to the CUDA runtime
    assert len(alloc.live) == 1
    ctx.close()
    assert not alloc.live


def test_dependency_wait_runs_out_and_context_recovers(cuda_lib, restatement):
    m = _chain(1_000_000)
    rng = np.random.default_rng(9)
    b0 = rng.uniform(-1, 1, m.rows)
    ctx = context()
    a = csr(m.rows, m.cols, m.ptr, m.idx, m.val)
    assert ctx.device_status(clear=True) == 0
    ctx.check(ctx._lib.asc_sb_context_set_wait_limit(ctx.handle, 1))
    b = dev(b0)
    CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kLower,
                              SparseBlasDiagonal.kNonUnit, vec(b))
    torch.cuda.synchronize()
    assert ctx.device_status(clear=True) == 1  # a wait gave up; the launch ended
    with pytest.raises(AscError) as err:
        ctx.check(ctx._lib.asc_sb_context_set_wait_limit(ctx.handle, -1))
    assert err.value.code == ErrorCode.kInvalidArgument
    ctx.check(ctx._lib.asc_sb_context_set_wait_limit(ctx.handle, 0))  # back to 2 s
    b = dev(b0)
    CudaSparseTriangularSolve(ctx, SparseBlasTranspose.kNone, 1.0, a, SparseBlasTriangle.kLower,
                              SparseBlasDiagonal.kNonUnit, vec(b))
    want = restatement.triangular_solve(OP_NONE, 1, 0, m.rows, m.ptr, m.idx, m.val, 1.0,
                                        b0.reshape(-1, 1).copy(), 1, None, 1)
    assert bits_equal(host(b), want.reshape(-1))
    assert ctx.device_status() == 0
    ctx.close()
