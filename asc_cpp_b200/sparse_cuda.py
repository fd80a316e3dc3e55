"""Python mirror of ASCCpp's ``sparse_cuda`` facet over the C ABI.

Names, argument meaning and error behaviour follow the reference's public
templates in include/asc/sparse/providers/cuda.h:

* :class:`SparseCudaContext` - ``SparseCudaContext::Create`` (cuda.h:514).
* :func:`CudaCloneCsr` - ``CudaCloneCsr`` (cuda.h:1040-1056): copies a host
  CSR matrix to device memory and returns a trusted device array.
* :class:`CudaStridedVectorView` - cuda.h:616-730 (stride may also be negative
  here, as ``SparseBlasVectorView`` allows for the standard entry points).
* :func:`CudaCsrSpmvWorkspaceSize` / :func:`CudaCsrSpmv` - cuda.h:1758-1802.
* :func:`CudaSpmv` / :func:`CudaSpmm` - cuda.h:1616-1658.

Every failing call raises :class:`AscError` carrying the reference's
``ErrorCode``; like the reference, a failing call has not enqueued anything.
Device memory and streams come from torch (plumbing only); every kernel runs in
``libasc_sparse_b200.so``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._abi import (Determinism, ElementKind, ErrorCode, FormatKind,
                   MemorySpace, SparseBlasLayout, SparseBlasTranspose,
                   Variant)


class AscError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ErrorCode(code).name}: {message}")
        self.code = ErrorCode(code)
        self.message = message


def _kind(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return ElementKind.kDouble
    if dtype == torch.float32:
        return ElementKind.kFloat
    if dtype == torch.complex64:
        return ElementKind.kComplexFloat
    if dtype == torch.complex128:
        return ElementKind.kComplexDouble
    raise TypeError(f"unsupported element type {dtype}")


class SparseCudaContext:
    """Owns a library context bound to one device and one CUDA stream."""

    def __init__(self, handle: int, device: int, stream):
        self._lib = _abi.load()
        self._h = ctypes.c_void_p(handle)
        self.device = device
        self._stream = stream

    @classmethod
    def Create(cls, device: int = 0, stream: torch.cuda.Stream | None = None,
               determinism: Determinism = Determinism.kDeterministic
               ) -> "SparseCudaContext":
        lib = _abi.load()
        if stream is None:
            with torch.cuda.device(device):
                stream = torch.cuda.Stream(device=device)
        h = ctypes.c_void_p()
        # handle 0 is torch's legacy default stream: pass cudaStreamLegacy (0x1),
        # because a NULL stream asks the library to create its own.
        raw = stream.cuda_stream or 1
        rc = lib.asc_sb_context_create(device, ctypes.c_void_p(raw), ctypes.byref(h))
        if rc != 0:
            raise AscError(rc, "could not create the sparse CUDA context")
        ctx = cls(h.value, device, stream)
        ctx.set_determinism(determinism)
        return ctx

    # -- handle management --
    @property
    def handle(self) -> ctypes.c_void_p:
        if self._h is None or not self._h.value:
            raise AscError(ErrorCode.kInvalidState,
                           "A moved-from SparseCudaContext cannot launch work")
        return self._h

    def close(self) -> None:
        if self._h is not None and self._h.value:
            self._lib.asc_sb_context_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self) -> torch.cuda.Stream:
        return self._stream

    def check(self, rc: int) -> None:
        if rc != 0:
            msg = self._lib.asc_sb_context_last_error(self._h)
            raise AscError(rc, msg.decode() if msg else "")

    def set_determinism(self, determinism: Determinism) -> None:
        self.check(self._lib.asc_sb_context_set_determinism(self.handle, int(determinism)))

    def set_variant(self, variant: Variant, lanes: int = 0) -> None:
        self.check(self._lib.asc_sb_context_set_variant(self.handle, int(variant), lanes))

    def synchronize(self) -> None:
        self.check(self._lib.asc_sb_context_synchronize(self.handle))

    @property
    def launch_count(self) -> int:
        return int(self._lib.asc_sb_context_launch_count(self.handle))

    def device_status(self, clear: bool = False) -> int:
        """Nonzero if a kernel of this context gave up a bounded wait."""
        v = ctypes.c_int32()
        self.check(self._lib.asc_sb_context_device_status(self.handle, ctypes.byref(v),
                                                          1 if clear else 0))
        return v.value


@dataclass
class CudaCsrArray:
    """Trusted device CSR (or CSC) matrix: int64 offsets/indices + values."""
    rows: int
    columns: int
    offsets: torch.Tensor
    indices: torch.Tensor
    values: torch.Tensor
    format: FormatKind = FormatKind.kCsr

    @property
    def nnz(self) -> int:
        return int(self.indices.numel())

    def describe(self) -> _abi.SparseDesc:
        d = _abi.SparseDesc()
        d.structure_first = self.offsets.data_ptr()
        d.structure_second = self.indices.data_ptr() if self.nnz else None
        d.values = self.values.data_ptr() if self.nnz else None
        d.memory_space = MemorySpace.kDevice
        d.element_kind = _kind(self.values.dtype)
        d.format = int(self.format)
        d.canonical_structure_trusted = 1
        d.rows = self.rows
        d.columns = self.columns
        d.nonzeros = self.nnz
        return d


def _host_sparse_desc(rows, columns, offsets, indices, values, fmt) -> _abi.SparseDesc:
    d = _abi.SparseDesc()
    pinned = isinstance(values, torch.Tensor) and values.is_pinned()
    d.structure_first = _host_ptr(offsets)
    d.structure_second = _host_ptr(indices) if len(indices) else None
    d.values = _host_ptr(values) if len(values) else None
    d.memory_space = MemorySpace.kPinnedHost if pinned else MemorySpace.kHost
    d.element_kind = _kind(values.dtype if isinstance(values, torch.Tensor)
                           else torch.from_numpy(values[:0]).dtype)
    d.format = int(fmt)
    d.canonical_structure_trusted = 1
    d.rows, d.columns, d.nonzeros = rows, columns, len(values)
    return d


def _host_ptr(a) -> int:
    return a.data_ptr() if isinstance(a, torch.Tensor) else a.ctypes.data


def CudaCloneCsr(context: SparseCudaContext, rows: int, columns: int,
                 offsets, indices, values,
                 fmt: FormatKind = FormatKind.kCsr) -> CudaCsrArray:
    """Host CSR -> trusted device CSR (cuda.h:1040-1056) through
    asc_sb_clone_csr: device arrays allocated here (the caller's resource in
    the reference), copies on the context stream, pageable sources staged
    through pinned buffers.  Arrays are numpy arrays or (pinned) CPU tensors;
    the structure must already be canonical."""
    if not isinstance(offsets, torch.Tensor):
        offsets = np.ascontiguousarray(offsets, np.int64)
        indices = np.ascontiguousarray(indices, np.int64)
        values = np.ascontiguousarray(values)
    dev = torch.device("cuda", context.device)
    vdtype = values.dtype if isinstance(values, torch.Tensor) else \
        torch.from_numpy(values[:0]).dtype
    off = torch.empty(len(offsets), dtype=torch.int64, device=dev)
    idx = torch.empty(len(indices), dtype=torch.int64, device=dev)
    val = torch.empty(len(values), dtype=vdtype, device=dev)
    out = CudaCsrArray(rows, columns, off, idx, val, fmt)
    src = _host_sparse_desc(rows, columns, offsets, indices, values, fmt)
    dst = out.describe()
    context.check(context._lib.asc_sb_clone_csr(context.handle, ctypes.byref(src),
                                                ctypes.byref(dst)))
    return out


def CudaCloneIndexedVector(context: SparseCudaContext, indices, values,
                           dense_extent: int) -> tuple[torch.Tensor, torch.Tensor]:
    """Host indexed vector -> device (CloneIndexedErased semantics):
    returns the device (indices, values)."""
    from ._abi import IndexedDesc
    if not isinstance(indices, torch.Tensor):
        indices = np.ascontiguousarray(indices, np.int64)
        values = np.ascontiguousarray(values)
    dev = torch.device("cuda", context.device)
    vdtype = values.dtype if isinstance(values, torch.Tensor) else \
        torch.from_numpy(values[:0]).dtype
    d_idx = torch.empty(len(indices), dtype=torch.int64, device=dev)
    d_val = torch.empty(len(values), dtype=vdtype, device=dev)
    s, d = IndexedDesc(), IndexedDesc()
    pinned = isinstance(values, torch.Tensor) and values.is_pinned()
    s.indices = _host_ptr(indices) if len(indices) else None
    s.values = _host_ptr(values) if len(values) else None
    s.memory_space = MemorySpace.kPinnedHost if pinned else MemorySpace.kHost
    d.indices = d_idx.data_ptr() if len(indices) else None
    d.values = d_val.data_ptr() if len(values) else None
    d.memory_space = MemorySpace.kDevice
    for x in (s, d):
        x.element_kind = _kind(vdtype)
        x.nonzeros = len(values)
        x.dense_extent = dense_extent
        x.writable = 1
        x.canonical_structure_trusted = 1
    context.check(context._lib.asc_sb_clone_indexed(context.handle, ctypes.byref(s),
                                                    ctypes.byref(d)))
    return d_idx, d_val


@dataclass
class CudaStridedVectorView:
    """``extent`` elements of ``tensor`` starting at element ``offset`` with
    ``stride``; logical element i is storage element offset + i*stride."""
    tensor: torch.Tensor
    extent: int
    stride: int = 1
    offset: int = 0
    writable: bool = True

    @classmethod
    def of(cls, t: torch.Tensor, writable: bool = True) -> "CudaStridedVectorView":
        return cls(t, t.numel(), 1, 0, writable)

    def describe(self) -> _abi.VectorDesc:
        d = _abi.VectorDesc()
        es = self.tensor.element_size()
        d.data = self.tensor.data_ptr() + self.offset * es if self.extent else None
        d.reachable_data = None
        d.reachable_size = 0
        d.memory_space = (MemorySpace.kDevice if self.tensor.is_cuda
                          else MemorySpace.kHost)
        d.element_kind = _kind(self.tensor.dtype)
        d.extent = self.extent
        d.stride = self.stride
        d.writable = 1 if self.writable else 0
        return d


@dataclass
class DenseMatrixView:
    tensor: torch.Tensor
    rows: int
    columns: int
    layout: SparseBlasLayout = SparseBlasLayout.kRowMajor
    leading_dimension: int | None = None
    writable: bool = True

    def describe(self) -> _abi.DenseDesc:
        d = _abi.DenseDesc()
        d.data = self.tensor.data_ptr()
        d.reachable_data = None
        d.reachable_size = 0
        d.memory_space = MemorySpace.kDevice if self.tensor.is_cuda else MemorySpace.kHost
        d.element_kind = _kind(self.tensor.dtype)
        d.rows = self.rows
        d.columns = self.columns
        if self.leading_dimension is None:
            ld = self.columns if self.layout == SparseBlasLayout.kRowMajor else self.rows
            ld = max(ld, 1)
        else:
            ld = self.leading_dimension
        d.leading_dimension = ld
        d.layout = int(self.layout)
        d.writable = 1 if self.writable else 0
        return d


def CudaCsrSpmvWorkspaceSize(context: SparseCudaContext, matrix: CudaCsrArray,
                             x: CudaStridedVectorView,
                             y: CudaStridedVectorView) -> int:
    n = ctypes.c_size_t()
    m, xd, yd = matrix.describe(), x.describe(), y.describe()
    xd.writable = 0
    context.check(context._lib.asc_sb_csr_spmv_workspace_size(
        context.handle, ctypes.byref(m), ctypes.byref(xd), ctypes.byref(yd), ctypes.byref(n)))
    return n.value


def CudaCsrSpmv(context: SparseCudaContext, alpha: float, matrix: CudaCsrArray,
                x: CudaStridedVectorView, beta: float, y: CudaStridedVectorView,
                workspace: torch.Tensor | None = None,
                workspace_bytes: int | None = None,
                workspace_space: MemorySpace | None = None) -> None:
    """y = alpha*A*x + beta*y, enqueued on the context stream.  The workspace
    placement defaults to where the workspace tensor lives."""
    m, xd, yd = matrix.describe(), x.describe(), y.describe()
    xd.writable = 0
    if workspace_space is None:
        workspace_space = (MemorySpace.kHost if workspace is not None and not workspace.is_cuda
                           else MemorySpace.kDevice)
    if workspace is None:
        wptr, wbytes = None, 0 if workspace_bytes is None else workspace_bytes
    else:
        wptr = workspace.data_ptr()
        wbytes = workspace.numel() * workspace.element_size() if workspace_bytes is None \
            else workspace_bytes
    context.check(context._lib.asc_sb_csr_spmv(
        context.handle, float(alpha), ctypes.byref(m), ctypes.byref(xd), float(beta),
        ctypes.byref(yd), wptr, wbytes, int(workspace_space)))


def CudaSpmv(context: SparseCudaContext, op: SparseBlasTranspose, alpha: float,
             matrix: CudaCsrArray, x: CudaStridedVectorView,
             y: CudaStridedVectorView, plan: "CsrPlan | None" = None) -> None:
    """y += alpha*op(A)*x (blas.h:1607-1667 semantics)."""
    m, xd, yd = matrix.describe(), x.describe(), y.describe()
    xd.writable = 0
    a = complex(alpha)
    if plan is not None:
        context.check(context._lib.asc_sb_plan_standard_spmv(
            context.handle, plan.handle, int(op), a.real, a.imag, ctypes.byref(xd),
            ctypes.byref(yd)))
        return
    context.check(context._lib.asc_sb_standard_spmv(
        context.handle, int(op), a.real, a.imag, ctypes.byref(m), ctypes.byref(xd),
        ctypes.byref(yd)))


def CudaSpmm(context: SparseCudaContext, op: SparseBlasTranspose, alpha: float,
             matrix: CudaCsrArray, b: DenseMatrixView, c: DenseMatrixView,
             plan: "CsrPlan | None" = None) -> None:
    """C += alpha*op(A)*B (blas.h:1692-1750 semantics)."""
    m, bd, cd = matrix.describe(), b.describe(), c.describe()
    bd.writable = 0
    a = complex(alpha)
    if plan is not None:
        context.check(context._lib.asc_sb_plan_standard_spmm(
            context.handle, plan.handle, int(op), a.real, a.imag, ctypes.byref(bd),
            ctypes.byref(cd)))
        return
    context.check(context._lib.asc_sb_standard_spmm(
        context.handle, int(op), a.real, a.imag, ctypes.byref(m), ctypes.byref(bd),
        ctypes.byref(cd)))


def CudaSparseTriangularSolveMultiple(context: SparseCudaContext, op: SparseBlasTranspose,
                                      alpha: complex, matrix: CudaCsrArray, triangle: int,
                                      diagonal: int, right_hand_sides: DenseMatrixView,
                                      plan: "CsrPlan | None" = None) -> None:
    """Solves op(A) X = alpha B in place (cuda.h:1727-1739 /
    blas.h:1856-1910 semantics); with a plan, its triangular-solve state and
    transposed structure are used."""
    rd = right_hand_sides.describe()
    a = complex(alpha)
    if plan is not None:
        context.check(context._lib.asc_sb_plan_triangular_solve(
            context.handle, plan.handle, int(op), a.real, a.imag, int(triangle), int(diagonal),
            ctypes.byref(rd)))
        return
    m = matrix.describe()
    context.check(context._lib.asc_sb_standard_triangular_solve(
        context.handle, int(op), a.real, a.imag, ctypes.byref(m), int(triangle), int(diagonal),
        ctypes.byref(rd)))


def CudaSparseTriangularSolve(context: SparseCudaContext, op: SparseBlasTranspose,
                              alpha: complex, matrix: CudaCsrArray, triangle: int,
                              diagonal: int, right_hand_side: CudaStridedVectorView,
                              plan: "CsrPlan | None" = None) -> None:
    """One right-hand side (cuda.h:1680-1705): the vector is passed as an
    n x 1 row-major matrix whose leading dimension is its increment."""
    v = right_hand_side
    es = v.tensor.element_size()
    view = DenseMatrixView(v.tensor, v.extent, 1, SparseBlasLayout.kRowMajor, v.stride,
                           v.writable)
    rd = view.describe()
    rd.data = v.tensor.data_ptr() + v.offset * es if v.extent else None
    a = complex(alpha)
    if plan is not None:
        context.check(context._lib.asc_sb_plan_triangular_solve(
            context.handle, plan.handle, int(op), a.real, a.imag, int(triangle), int(diagonal),
            ctypes.byref(rd)))
        return
    m = matrix.describe()
    context.check(context._lib.asc_sb_standard_triangular_solve(
        context.handle, int(op), a.real, a.imag, ctypes.byref(m), int(triangle), int(diagonal),
        ctypes.byref(rd)))


class CsrPlan:
    """Cached analysis of one device matrix (partitions, transposed structure),
    stored in a device buffer this object owns."""

    def __init__(self, context: SparseCudaContext, matrix: CudaCsrArray,
                 flags: int = 0):
        self.context = context
        self.matrix = matrix
        d = matrix.describe()
        n = ctypes.c_size_t()
        context.check(context._lib.asc_sb_plan_workspace_size(
            context.handle, ctypes.byref(d), flags, ctypes.byref(n)))
        self.buffer = torch.empty(max(n.value, 1), dtype=torch.uint8,
                                  device=torch.device("cuda", context.device))
        h = ctypes.c_void_p()
        context.check(context._lib.asc_sb_plan_create(
            context.handle, ctypes.byref(d), flags, self.buffer.data_ptr(), n.value,
            ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def properties(self) -> int:
        """Bit set of ASC_SB_PLAN_HAS_TRANSPOSE / ASC_SB_PLAN_HAS_BLOCKS16."""
        v = ctypes.c_int32()
        self.context.check(self.context._lib.asc_sb_plan_properties(self._h, ctypes.byref(v)))
        return v.value

    def triangular_analysis(self, op: SparseBlasTranspose, triangle: int) -> None:
        """Level order for solves with this op class and triangle (plans
        created with ASC_SB_PLAN_TRIANGULAR)."""
        self.context.check(self.context._lib.asc_sb_plan_triangular_analysis(
            self.context.handle, self._h, int(op), int(triangle)))

    def refresh_values(self) -> None:
        """Re-gathers the transposed values after the matrix's values changed."""
        self.context.check(self.context._lib.asc_sb_plan_refresh_values(
            self.context.handle, self._h))

    def spmm_autotune(self, alpha: float, b: "DenseMatrixView", c: "DenseMatrixView",
                      reps: int = 5) -> tuple[float, int]:
        """Times the SpMM kernels on these operands (C accumulates) and keeps
        the fastest; returns (ms per product, rows per group: 0 = row by row,
        SPMM_STAGED = the TMA-staged kernel).  Needs a plan created with
        PLAN_ROW_GROUPS."""
        bd, cd = b.describe(), c.describe()
        bd.writable = 0
        ms = ctypes.c_float()
        rg = ctypes.c_int32()
        self.context.check(self.context._lib.asc_sb_plan_spmm_autotune(
            self.context.handle, self._h, float(alpha), ctypes.byref(bd), ctypes.byref(cd),
            reps, ctypes.byref(ms), ctypes.byref(rg)))
        return ms.value, rg.value

    def set_spmm(self, choice: int) -> None:
        """Chooses the SpMM kernel: 0 row by row, SPMM_STAGED, R rows per
        group (2..32), or SPMM_AUTO.  Needs a plan created with
        PLAN_ROW_GROUPS."""
        self.context.check(self.context._lib.asc_sb_plan_set_spmm(self.context.handle, self._h,
                                                                   int(choice)))

    def spmm_stage_rows(self, k: int) -> int:
        """Rows per group of the staged SpMM tables a product with k columns
        (row-major, leading dimension k) would use: 16, 32, 64 or 0."""
        rows = ctypes.c_int64()
        self.context.check(self.context._lib.asc_sb_plan_spmm_stage_rows(
            self.context.handle, self._h, int(k), ctypes.byref(rows)))
        return int(rows.value)

    def spmm_tuning(self) -> dict[int, float]:
        """The last spmm_autotune's table: {candidate: ms per product}."""
        count = ctypes.c_int32()
        cands = (ctypes.c_int32 * 8)()
        ms = (ctypes.c_float * 8)()
        rc = self.context._lib.asc_sb_plan_spmm_tuning(self._h, 8, ctypes.byref(count), cands, ms)
        if rc != 0:
            raise AscError(rc, "asc_sb_plan_spmm_tuning failed")
        return {int(cands[i]): float(ms[i]) for i in range(min(count.value, 8))}

    def csr_spmv(self, alpha: float, x: CudaStridedVectorView, beta: float,
                 y: CudaStridedVectorView) -> None:
        xd, yd = x.describe(), y.describe()
        xd.writable = 0
        self.context.check(self.context._lib.asc_sb_plan_csr_spmv(
            self.context.handle, self._h, float(alpha), ctypes.byref(xd), float(beta),
            ctypes.byref(yd)))

    def close(self):
        if self._h is not None and self._h.value:
            self.context._lib.asc_sb_plan_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- format conversion on the device (compressed.h:1082-1221 semantics) ----

def _convert_workspace(context: SparseCudaContext, rows: int, columns: int, nnz: int,
                       fmt: FormatKind) -> torch.Tensor:
    n = ctypes.c_size_t()
    context.check(context._lib.asc_sb_convert_workspace_size(
        context.handle, rows, columns, nnz, int(fmt), ctypes.byref(n)))
    return torch.empty(max(n.value, 1), dtype=torch.uint8,
                       device=torch.device("cuda", context.device))


def _empty_compressed(context: SparseCudaContext, rows: int, columns: int, nnz: int,
                      dtype: torch.dtype, fmt: FormatKind) -> CudaCsrArray:
    dev = torch.device("cuda", context.device)
    outer = rows if fmt == FormatKind.kCsr else columns
    return CudaCsrArray(rows, columns, torch.empty(outer + 1, dtype=torch.int64, device=dev),
                        torch.empty(nnz, dtype=torch.int64, device=dev),
                        torch.empty(nnz, dtype=dtype, device=dev), fmt)


def CudaConvertCompressed(context: SparseCudaContext, source: CudaCsrArray) -> CudaCsrArray:
    """CSR -> CSC or CSC -> CSR of the same matrix, on the device
    (ConvertToCsc(CsrView) / ConvertToCsr(CscView), compressed.h:1728-1780)."""
    fmt = FormatKind.kCsc if source.format == FormatKind.kCsr else FormatKind.kCsr
    with torch.cuda.stream(context.stream):
        out = _empty_compressed(context, source.rows, source.columns, source.nnz,
                                source.values.dtype, fmt)
        ws = _convert_workspace(context, source.rows, source.columns, source.nnz, fmt)
    sd, dd = source.describe(), out.describe()
    dd.canonical_structure_trusted = 0
    context.check(context._lib.asc_sb_convert_compressed(
        context.handle, ctypes.byref(sd), ctypes.byref(dd), ws.data_ptr(), ws.numel()))
    ws.record_stream(context.stream)
    return out


def CudaConvertCoordinates(context: SparseCudaContext, rows: int, columns: int,
                           coordinates: torch.Tensor, values: torch.Tensor,
                           fmt: FormatKind = FormatKind.kCsr) -> CudaCsrArray:
    """Device (row, column) pairs [nnz, 2] + values -> CSR or CSC
    (ConvertToCsr / ConvertToCsc(CoordinateView), compressed.h:1676-1726)."""
    nnz = int(values.numel())
    with torch.cuda.stream(context.stream):
        out = _empty_compressed(context, rows, columns, nnz, values.dtype, fmt)
        ws = _convert_workspace(context, rows, columns, nnz, fmt)
    dd = out.describe()
    dd.canonical_structure_trusted = 0
    context.check(context._lib.asc_sb_convert_coordinates(
        context.handle, coordinates.data_ptr() if nnz else None,
        values.data_ptr() if nnz else None, _kind(values.dtype), rows, columns, nnz,
        ctypes.byref(dd), ws.data_ptr(), ws.numel()))
    ws.record_stream(context.stream)
    return out


# ---- batched SpMV (one persistent launch for many matrices) ----

class CudaBatch:
    """Binds independent products y_i = alpha*A_i*x_i + beta*y_i and runs them
    as one persistent launch (asc_sb_batch_*)."""

    def __init__(self, context: SparseCudaContext, matrices: list[CudaCsrArray],
                 inputs: list[CudaStridedVectorView], outputs: list[CudaStridedVectorView]):
        self.context = context
        self._keep = (matrices, inputs, outputs)
        n = len(matrices)
        mats = (_abi.SparseDesc * max(n, 1))(*[m.describe() for m in matrices])
        xs = (_abi.VectorDesc * max(n, 1))(*[x.describe() for x in inputs])
        ys = (_abi.VectorDesc * max(n, 1))(*[y.describe() for y in outputs])
        for i in range(n):
            xs[i].writable = 0
        size = ctypes.c_size_t()
        lib = context._lib
        context.check(lib.asc_sb_batch_workspace_size(context.handle, n, mats,
                                                      ctypes.byref(size)))
        self.workspace = torch.empty(max(size.value, 256), dtype=torch.uint8,
                                     device=torch.device("cuda", context.device))
        h = ctypes.c_void_p()
        context.check(lib.asc_sb_batch_create(context.handle, n, mats, xs, ys,
                                              self.workspace.data_ptr(), size.value,
                                              ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def spmv(self, alpha: float, beta: float) -> None:
        self.context.check(self.context._lib.asc_sb_batch_spmv(
            self.context.handle, self._h, float(alpha), float(beta)))

    def spmv_per_matrix(self, alpha: float, beta: float) -> None:
        self.context.check(self.context._lib.asc_sb_batch_spmv_per_matrix(
            self.context.handle, self._h, float(alpha), float(beta)))

    def capture(self, alpha: float, beta: float) -> None:
        self.context.check(self.context._lib.asc_sb_batch_capture(
            self.context.handle, self._h, float(alpha), float(beta)))

    def set_schedule(self, chunk_tiles: int, ctas_per_sm: int = 0) -> None:
        self.context.check(self.context._lib.asc_sb_batch_set_schedule(
            self.context.handle, self._h, int(chunk_tiles), int(ctas_per_sm)))

    def schedule(self) -> tuple[int, int]:
        c, k = ctypes.c_int32(), ctypes.c_int32()
        rc = self.context._lib.asc_sb_batch_get_schedule(self._h, ctypes.byref(c),
                                                         ctypes.byref(k))
        self.context.check(rc)
        return c.value, k.value

    def autotune(self, alpha: float, beta: float, reps: int = 3) -> float:
        best = ctypes.c_float()
        self.context.check(self.context._lib.asc_sb_batch_autotune(
            self.context.handle, self._h, float(alpha), float(beta), int(reps),
            ctypes.byref(best)))
        return best.value

    def close(self) -> None:
        if self._h is not None and self._h.value:
            self.context._lib.asc_sb_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- Level-1 on an indexed vector (blas.h:1340-1600 semantics) ----

def CudaLevel1(context: SparseCudaContext, operation: int, indices: torch.Tensor,
               values: torch.Tensor, dense: CudaStridedVectorView,
               result: torch.Tensor | None = None, alpha: complex = 0.0,
               conjugated: bool = False) -> None:
    """dot (result[0]), axpy, gather, gather-zero or scatter between the
    indexed vector (indices, values) and `dense` (internal_sparse_cuda::
    StandardLevel1Erased)."""
    from ._abi import IndexedDesc, Level1Op
    op = int(operation)
    d = IndexedDesc()
    d.indices = indices.data_ptr() if indices.numel() else None
    d.values = values.data_ptr() if values.numel() else None
    d.memory_space = MemorySpace.kDevice
    d.element_kind = _kind(values.dtype)
    d.nonzeros = int(values.numel())
    d.dense_extent = dense.extent
    d.writable = 1 if op in (Level1Op.kGather, Level1Op.kGatherZero) else 0
    d.canonical_structure_trusted = 1
    dd = dense.describe()
    dd.writable = 1 if op in (Level1Op.kAxpy, Level1Op.kGatherZero, Level1Op.kScatter) else 0
    rd = None
    if op == Level1Op.kDot:
        rd = CudaStridedVectorView(result, 1).describe()
    a = complex(alpha)
    context.check(context._lib.asc_sb_standard_level1(
        context.handle, op, 1 if conjugated else 0, a.real, a.imag, ctypes.byref(d),
        ctypes.byref(dd), ctypes.byref(rd) if rd is not None else None))
