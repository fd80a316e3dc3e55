"""CPU oracle for the Sparse BLAS hot path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``asc_cpp_b200``) never imports it.

Two backends:

* :class:`Restatement` - ``liboracle.so``, the C restatement in
  ``sparse_oracle.c`` (always available once built).
* :class:`Reference` - ``_ref/libasc_ref.so``, the reference's own serial
  Sparse BLAS compiled from its sources (present where it could be built).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build_oracle

_HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_INT = ctypes.c_int
_SZ = ctypes.c_size_t

CSR, CSC = 1, 2
OP_NONE, OP_TRANSPOSE, OP_CONJ_TRANSPOSE = 0, 1, 2
COL_MAJOR, ROW_MAJOR = 0, 1


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


def _scalar(dtype):
    return ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float


def _complex_suffix(dtype) -> str | None:
    dt = np.dtype(dtype)
    if dt == np.complex128:
        return "z"
    if dt == np.complex64:
        return "c"
    return None


def _real_scalar(dtype):
    return ctypes.c_double if np.dtype(dtype) == np.complex128 else ctypes.c_float


def _suffix(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"oracle supports float32/float64, not {dt}")


class Restatement:
    """ctypes front end of ``liboracle.so``."""

    def __init__(self, path: str | None = None):
        path = path or build_oracle.ORACLE_SO
        if not os.path.exists(path):
            build_oracle.build_restatement()
        self.lib = ctypes.CDLL(path)
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_compat_spmv_{sfx}")
            f.restype = None
            f.argtypes = [_I64, _P, _P, _P, sc, _P, _I64, sc, _P, _I64]
            f = getattr(self.lib, f"oracle_standard_spmv_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, sc, _P, _I64, _P,
                          _I64]
            f = getattr(self.lib, f"oracle_standard_spmm_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, sc, _P, _INT, _I64,
                          _P, _INT, _I64, _I64]
            f = getattr(self.lib, f"oracle_csr_extended_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _I64, _I64, _P, _P, _P, _P, _P, _P]
        for sfx, sc in (("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_complex_spmv_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, sc, sc, _P, _I64,
                          _P, _I64]
            f = getattr(self.lib, f"oracle_complex_spmm_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, sc, sc, _P, _INT,
                          _I64, _P, _INT, _I64, _I64]
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_level1_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _P, _P, _I64, sc, _P, _P]
        for sfx, sc in (("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_level1_{sfx}")
            f.restype = None
            f.argtypes = [_INT, _INT, _P, _P, _I64, sc, sc, _P, _P]
        self.lib.oracle_output_counts.restype = None
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_trsv_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _INT, _I64, _P, _P, _P, sc, _P, _INT, _I64, _I64]
        for sfx, sc in (("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"oracle_trsv_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _INT, _I64, _P, _P, _P, sc, sc, _P, _INT, _I64, _I64]
        self.lib.oracle_output_counts.argtypes = [_INT, _I64, _I64, _P, _P, _P]
        self.lib.oracle_csr_transpose_structure.restype = None
        self.lib.oracle_csr_transpose_structure.argtypes = [_I64, _I64, _P, _P,
                                                            _P, _P, _P]
        self.lib.oracle_stable_bucket_sort.restype = None
        self.lib.oracle_stable_bucket_sort.argtypes = [_I64, _P, _I64, _I64,
                                                       _P, _P]
        self.lib.oracle_merge_path_split.restype = None
        self.lib.oracle_merge_path_split.argtypes = [
            _I64, _P, _I64, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]

    # -- compat y = alpha*A*x + beta*y (strided; x, y point at element 0) --
    def compat_spmv(self, ptr, idx, val, alpha, x, beta, y, incx=1, incy=1):
        rows = len(ptr) - 1
        sc = _scalar(val.dtype)
        getattr(self.lib, f"oracle_compat_spmv_{_suffix(val.dtype)}")(
            rows, _ptr(ptr), _ptr(idx), _ptr(val), sc(alpha), _ptr(x), incx,
            sc(beta), _ptr(y), incy)
        return y

    def standard_spmv(self, fmt, op, rows, cols, ptr, idx, val, alpha, x, y,
                      incx=1, incy=1, x_offset=0, y_offset=0):
        """y += alpha*op(A)*x; ``*_offset`` = element index of logical 0."""
        xs = x.ctypes.data + x_offset * x.itemsize
        ys = y.ctypes.data + y_offset * y.itemsize
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            getattr(self.lib, f"oracle_complex_spmv_{cs}")(
                fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), rs(a.real),
                rs(a.imag), xs, incx, ys, incy)
            return y
        sc = _scalar(val.dtype)
        getattr(self.lib, f"oracle_standard_spmv_{_suffix(val.dtype)}")(
            fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), sc(alpha), xs,
            incx, ys, incy)
        return y

    def standard_spmm(self, fmt, op, rows, cols, ptr, idx, val, alpha, b,
                      b_layout, ldb, c, c_layout, ldc, ncols):
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            getattr(self.lib, f"oracle_complex_spmm_{cs}")(
                fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), rs(a.real),
                rs(a.imag), _ptr(b), b_layout, ldb, _ptr(c), c_layout, ldc, ncols)
            return c
        sc = _scalar(val.dtype)
        getattr(self.lib, f"oracle_standard_spmm_{_suffix(val.dtype)}")(
            fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), sc(alpha),
            _ptr(b), b_layout, ldb, _ptr(c), c_layout, ldc, ncols)
        return c

    def extended(self, op, rows, cols, ptr, idx, val, x):
        """(exact sum, sum of |products|) per output of op(A)x, long double."""
        n_out = rows if op == OP_NONE else cols
        exact = np.zeros(n_out, dtype=np.longdouble)
        absval = np.zeros(n_out, dtype=np.longdouble)
        getattr(self.lib, f"oracle_csr_extended_{_suffix(val.dtype)}")(
            op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), _ptr(x),
            _ptr(exact), _ptr(absval))
        return exact, absval

    def output_counts(self, op, rows, cols, ptr, idx):
        n_out = rows if op == OP_NONE else cols
        counts = np.zeros(n_out, dtype=np.int64)
        self.lib.oracle_output_counts(op, rows, cols, _ptr(ptr), _ptr(idx),
                                      _ptr(counts))
        return counts

    def transpose_structure(self, rows, cols, ptr, idx):
        nnz = int(ptr[rows])
        t_ptr = np.zeros(cols + 1, dtype=np.int64)
        t_idx = np.zeros(max(nnz, 1), dtype=np.int64)
        perm = np.zeros(max(nnz, 1), dtype=np.int64)
        self.lib.oracle_csr_transpose_structure(rows, cols, _ptr(ptr),
                                                _ptr(idx), _ptr(t_ptr),
                                                _ptr(t_idx), _ptr(perm))
        return t_ptr, t_idx[:nnz], perm[:nnz]

    def level1(self, op, conj, idx, val, alpha, x):
        """Level-1 on copies: returns (values, dense, dot result)."""
        val = val.copy()
        x = x.copy()
        res = np.zeros(1, dtype=val.dtype)
        idx = np.ascontiguousarray(idx, np.int64)
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            getattr(self.lib, f"oracle_level1_{cs}")(op, conj, _ptr(idx), _ptr(val), len(idx),
                                                     rs(a.real), rs(a.imag), _ptr(x), _ptr(res))
        else:
            sc = _scalar(val.dtype)
            getattr(self.lib, f"oracle_level1_{_suffix(val.dtype)}")(
                op, conj, _ptr(idx), _ptr(val), len(idx), sc(float(np.real(alpha))), _ptr(x),
                _ptr(res))
        return val, x, res[0]

    def triangular_solve(self, op, triangle, diagonal, n, ptr, idx, val, alpha, b,
                         layout=ROW_MAJOR, ld=None, k=1):
        """Solves op(A) X = alpha B for square CSR A on a copy of the dense
        storage ``b`` (n x k, ``layout``, ``ld``); returns the copy."""
        b = np.array(b, copy=True)
        ld = (k if layout == ROW_MAJOR else n) if ld is None else ld
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            rc = getattr(self.lib, f"oracle_trsv_{cs}")(
                op, triangle, diagonal, n, _ptr(ptr), _ptr(idx), _ptr(val), rs(a.real),
                rs(a.imag), _ptr(b), layout, ld, k)
        else:
            sc = _scalar(val.dtype)
            rc = getattr(self.lib, f"oracle_trsv_{_suffix(val.dtype)}")(
                op, triangle, diagonal, n, _ptr(ptr), _ptr(idx), _ptr(val),
                sc(float(np.real(alpha))), _ptr(b), layout, ld, k)
        if rc != 0:
            raise MemoryError("oracle triangular solve could not allocate")
        return b

    def stable_bucket_sort(self, keys, kstride, n, limit):
        """(offsets[limit+1], perm[n]) of the stable sort of keys[e*kstride]."""
        offsets = np.zeros(limit + 1, dtype=np.int64)
        perm = np.zeros(max(n, 1), dtype=np.int64)
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        self.lib.oracle_stable_bucket_sort(n, _ptr(keys), kstride, limit,
                                           _ptr(offsets), _ptr(perm))
        return offsets, perm[:n]

    def convert_compressed(self, to_csc, rows, cols, ptr, idx, val):
        """CSR arrays -> CSC arrays (to_csc) or CSC -> CSR, stable order."""
        outer_in = rows if to_csc else cols
        outer_out = cols if to_csc else rows
        nnz = int(ptr[outer_in])
        offsets, perm = self.stable_bucket_sort(idx, 1, nnz, outer_out)
        source_outer = np.repeat(np.arange(outer_in, dtype=np.int64),
                                 np.diff(ptr))
        return offsets, source_outer[perm], val[perm]

    def convert_coordinates(self, to_csc, rows, cols, coordinates, val):
        """Interleaved [nnz][2] coordinates -> CSR (to_csc = 0) or CSC."""
        nnz = len(val)
        c = np.ascontiguousarray(coordinates, dtype=np.int64).reshape(-1)
        key = c[1:] if to_csc else c
        other = c[0::2] if to_csc else c[1::2]
        offsets, perm = self.stable_bucket_sort(key, 2, nnz,
                                                cols if to_csc else rows)
        return offsets, other[perm], val[perm]

    def merge_path_split(self, ptr, diagonal):
        rows = len(ptr) - 1
        r = _I64()
        z = _I64()
        self.lib.oracle_merge_path_split(rows, _ptr(ptr), int(ptr[-1]),
                                         int(diagonal), ctypes.byref(r),
                                         ctypes.byref(z))
        return r.value, z.value


class Reference:
    """ctypes front end of the reference's own serial Sparse BLAS."""

    def __init__(self, path: str | None = None):
        path = path or build_oracle.REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(self.lib, f"ref_compat_spmv_{sfx}")
            f.restype = _INT
            f.argtypes = [_I64, _I64, _P, _P, _P, _I64, sc, _P, _I64, sc, _P,
                          _I64]
            f = getattr(self.lib, f"ref_standard_spmv_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, _I64, sc, _P, _I64,
                          _I64, _SZ, _P, _I64, _I64, _SZ]
            f = getattr(self.lib, f"ref_standard_spmm_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, _I64, sc, _P, _I64,
                          _I64, _INT, _I64, _SZ, _P, _I64, _I64, _INT, _I64, _SZ]
            f = getattr(self.lib, f"ref_blocks_prepare_{sfx}")
            f.restype = _P
            f.argtypes = [_I64, _I64, _P, _P, _P, _INT]
            f = getattr(self.lib, f"ref_blocks_run_{sfx}")
            f.restype = _INT
            f.argtypes = [_P, sc, _P, sc, _P]
            f = getattr(self.lib, f"ref_blocks_free_{sfx}")
            f.restype = None
            f.argtypes = [_P]
        for sfx, sc in (("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"ref_standard_spmv_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, _I64, sc, sc, _P,
                          _I64, _I64, _SZ, _P, _I64, _I64, _SZ]
            f = getattr(self.lib, f"ref_standard_spmm_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _I64, _I64, _P, _P, _P, _I64, sc, sc, _P,
                          _I64, _I64, _INT, _I64, _SZ, _P, _I64, _I64, _INT,
                          _I64, _SZ]
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float),
                        ("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"ref_level1_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _P, _P, _I64, _I64, sc, sc, _P, _P]
        for sfx, sc in (("f64", ctypes.c_double), ("f32", ctypes.c_float),
                        ("z", ctypes.c_double), ("c", ctypes.c_float)):
            f = getattr(self.lib, f"ref_trsv_{sfx}")
            f.restype = _INT
            f.argtypes = [_INT, _INT, _INT, _I64, _P, _P, _P, _I64, sc, sc, _P, _INT, _I64,
                          _I64, _SZ]
        f = self.lib.ref_convert_compressed_f64
        f.restype = _INT
        f.argtypes = [_INT, _I64, _I64, _P, _P, _P, _I64, _P, _P, _P]
        f = self.lib.ref_convert_coordinates_f64
        f.restype = _INT
        f.argtypes = [_INT, _I64, _I64, _P, _P, _I64, _P, _P, _P]

    @staticmethod
    def available() -> bool:
        return os.path.exists(build_oracle.REF_SO)

    def compat_spmv(self, rows, cols, ptr, idx, val, alpha, x, beta, y,
                    incx=1, incy=1) -> int:
        sc = _scalar(val.dtype)
        return getattr(self.lib, f"ref_compat_spmv_{_suffix(val.dtype)}")(
            rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), int(ptr[rows]),
            sc(alpha), _ptr(x), incx, sc(beta), _ptr(y), incy)

    def standard_spmv(self, fmt, op, rows, cols, ptr, idx, val, alpha, x, y,
                      incx=1, incy=1, x_offset=0, y_offset=0) -> int:
        sc = _scalar(val.dtype)
        outer = rows if fmt == CSR else cols
        nx = cols if op == OP_NONE else rows
        ny = rows if op == OP_NONE else cols
        xs = x.ctypes.data + x_offset * x.itemsize
        ys = y.ctypes.data + y_offset * y.itemsize
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            return getattr(self.lib, f"ref_standard_spmv_{cs}")(
                fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val),
                int(ptr[outer]), rs(a.real), rs(a.imag), xs, nx, incx, x.size, ys,
                ny, incy, y.size)
        return getattr(self.lib, f"ref_standard_spmv_{_suffix(val.dtype)}")(
            fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val),
            int(ptr[outer]), sc(alpha), xs, nx, incx, x.size, ys, ny, incy,
            y.size)

    def standard_spmm(self, fmt, op, rows, cols, ptr, idx, val, alpha, b,
                      b_rows, b_cols, b_layout, ldb, c, c_rows, c_cols,
                      c_layout, ldc) -> int:
        outer = rows if fmt == CSR else cols
        cs = _complex_suffix(val.dtype)
        if cs is not None:
            rs = _real_scalar(val.dtype)
            a = complex(alpha)
            return getattr(self.lib, f"ref_standard_spmm_{cs}")(
                fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val),
                int(ptr[outer]), rs(a.real), rs(a.imag), _ptr(b), b_rows, b_cols,
                b_layout, ldb, b.size, _ptr(c), c_rows, c_cols, c_layout, ldc,
                c.size)
        sc = _scalar(val.dtype)
        return getattr(self.lib, f"ref_standard_spmm_{_suffix(val.dtype)}")(
            fmt, op, rows, cols, _ptr(ptr), _ptr(idx), _ptr(val),
            int(ptr[outer]), sc(alpha), _ptr(b), b_rows, b_cols, b_layout, ldb,
            b.size, _ptr(c), c_rows, c_cols, c_layout, ldc, c.size)

    # row-block parallel compat SpMV (each block is the reference's serial
    # SpmvReference on a disjoint row range)
    def blocks_prepare(self, rows, cols, ptr, idx, val, nblocks):
        h = getattr(self.lib, f"ref_blocks_prepare_{_suffix(val.dtype)}")(
            rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), nblocks)
        if not h:
            raise RuntimeError("reference rejected a row block")
        return h

    def blocks_run(self, h, dtype, alpha, x, beta, y) -> int:
        sc = _scalar(dtype)
        return getattr(self.lib, f"ref_blocks_run_{_suffix(dtype)}")(
            h, sc(alpha), _ptr(x), sc(beta), _ptr(y))

    def blocks_free(self, h, dtype) -> None:
        getattr(self.lib, f"ref_blocks_free_{_suffix(dtype)}")(h)

    # conversions (FP64 values), the reference's ConvertToCsr / ConvertToCsc
    def convert_compressed(self, to_csc, rows, cols, ptr, idx, val):
        outer_in = rows if to_csc else cols
        outer_out = cols if to_csc else rows
        nnz = int(ptr[outer_in])
        o = np.zeros(outer_out + 1, dtype=np.int64)
        i = np.zeros(max(nnz, 1), dtype=np.int64)
        v = np.zeros(max(nnz, 1), dtype=np.float64)
        rc = self.lib.ref_convert_compressed_f64(
            int(to_csc), rows, cols, _ptr(ptr), _ptr(idx), _ptr(val), nnz,
            _ptr(o), _ptr(i), _ptr(v))
        if rc != 0:
            raise RuntimeError(f"reference conversion failed with code {rc}")
        return o, i[:nnz], v[:nnz]

    def convert_coordinates(self, to_csc, rows, cols, coordinates, val):
        nnz = len(val)
        c = np.ascontiguousarray(coordinates, dtype=np.int64).reshape(-1)
        outer_out = cols if to_csc else rows
        o = np.zeros(outer_out + 1, dtype=np.int64)
        i = np.zeros(max(nnz, 1), dtype=np.int64)
        v = np.zeros(max(nnz, 1), dtype=np.float64)
        rc = self.lib.ref_convert_coordinates_f64(
            int(to_csc), rows, cols, _ptr(c), _ptr(val), nnz, _ptr(o), _ptr(i),
            _ptr(v))
        if rc != 0:
            raise RuntimeError(f"reference conversion failed with code {rc}")
        return o, i[:nnz], v[:nnz]

    def level1(self, op, conj, idx, val, alpha, x):
        """The reference's Level-1 on copies: (values, dense, dot result)."""
        val = val.copy()
        x = x.copy()
        res = np.zeros(1, dtype=val.dtype)
        idx = np.ascontiguousarray(idx, np.int64)
        sfx = _complex_suffix(val.dtype) or _suffix(val.dtype)
        rs = _real_scalar(val.dtype) if _complex_suffix(val.dtype) else _scalar(val.dtype)
        a = complex(alpha)
        rc = getattr(self.lib, f"ref_level1_{sfx}")(op, conj, _ptr(idx), _ptr(val), len(idx),
                                                    x.size, rs(a.real), rs(a.imag), _ptr(x),
                                                    _ptr(res))
        if rc != 0:
            raise RuntimeError(f"reference level-one failed with code {rc}")
        return val, x, res[0]

    def triangular_solve(self, op, triangle, diagonal, n, ptr, idx, val, alpha, b,
                         layout=ROW_MAJOR, ld=None, k=1):
        """The reference's SparseTriangularSolveMultiple on a copy of ``b``;
        returns (error code, solved copy)."""
        b = np.array(b, copy=True)
        ld = (k if layout == ROW_MAJOR else n) if ld is None else ld
        sfx = _complex_suffix(val.dtype) or _suffix(val.dtype)
        rs = _real_scalar(val.dtype) if _complex_suffix(val.dtype) else _scalar(val.dtype)
        a = complex(alpha)
        rc = getattr(self.lib, f"ref_trsv_{sfx}")(
            op, triangle, diagonal, n, _ptr(ptr), _ptr(idx), _ptr(val), int(ptr[n]),
            rs(a.real), rs(a.imag), _ptr(b), layout, ld, k, b.size)
        return rc, b


# ---- row-parallel drivers (full-size checks) --------------------------------
#
# For op = none every output row depends on that row's stored entries only,
# and the restatement walks each row in stored order, so running disjoint row
# blocks on separate threads gives the same bits as one serial call (ctypes
# releases the GIL for the duration of each call).

def _threads(threads: int | None) -> int:
    if threads:
        return threads
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(32, n))


def row_blocks(ptr: np.ndarray, parts: int) -> list[tuple[int, int]]:
    """Up to ``parts`` contiguous row blocks with about equal stored entries
    plus rows each."""
    rows = len(ptr) - 1
    if rows <= 0:
        return []
    weight_total = int(ptr[-1]) + rows
    cuts = [0]
    for k in range(1, parts):
        target = weight_total * k // parts
        # first row r with ptr[r] + r >= target
        lo, hi = cuts[-1], rows
        while lo < hi:
            mid = (lo + hi) // 2
            if int(ptr[mid]) + mid < target:
                lo = mid + 1
            else:
                hi = mid
        if lo > cuts[-1]:
            cuts.append(lo)
    cuts.append(rows)
    return [(a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]


def _run_blocks(fn, ptr, threads):
    from concurrent.futures import ThreadPoolExecutor
    blocks = row_blocks(ptr, 4 * _threads(threads))
    with ThreadPoolExecutor(max_workers=_threads(threads)) as ex:
        for f in [ex.submit(fn, r0, r1) for r0, r1 in blocks]:
            f.result()


def compat_spmv_rows(rs: "Restatement", ptr, idx, val, alpha, x, beta, y, threads=None):
    """Restatement.compat_spmv (unit strides) over row blocks in parallel."""
    _run_blocks(lambda r0, r1: rs.compat_spmv(ptr[r0:r1 + 1], idx, val, alpha, x, beta,
                                              y[r0:r1]), ptr, threads)
    return y


def standard_spmv_rows(rs: "Restatement", cols, ptr, idx, val, alpha, x, y, threads=None):
    """y += alpha*A*x (CSR, op none, unit strides) over row blocks in parallel."""
    _run_blocks(lambda r0, r1: rs.standard_spmv(CSR, OP_NONE, r1 - r0, cols, ptr[r0:r1 + 1],
                                                idx, val, alpha, x, y[r0:r1]), ptr, threads)
    return y


def standard_spmm_rows(rs: "Restatement", cols, ptr, idx, val, alpha, b, c, threads=None):
    """C += alpha*A*B (CSR, op none, row-major B [cols, k] and C [rows, k],
    contiguous) over row blocks in parallel."""
    k = b.shape[1]
    _run_blocks(lambda r0, r1: rs.standard_spmm(CSR, OP_NONE, r1 - r0, cols, ptr[r0:r1 + 1],
                                                idx, val, alpha, b, ROW_MAJOR, k, c[r0:r1],
                                                ROW_MAJOR, k, k), ptr, threads)
    return c


def extended_rows(rs: "Restatement", cols, ptr, idx, val, x, threads=None):
    """Restatement.extended for op none over row blocks in parallel: the
    long-double sum and sum of |products| of every row."""
    rows = len(ptr) - 1
    exact = np.zeros(rows, dtype=np.longdouble)
    absval = np.zeros(rows, dtype=np.longdouble)

    def part(r0, r1):
        e, a = rs.extended(OP_NONE, r1 - r0, cols, ptr[r0:r1 + 1], idx, val, x)
        exact[r0:r1] = e
        absval[r0:r1] = a
    _run_blocks(part, ptr, threads)
    return exact, absval


def gamma(n, dtype) -> np.ndarray:
    """gamma_n = n u / (1 - n u), u the unit roundoff of ``dtype``."""
    u = np.finfo(dtype).eps / 2
    n = np.asarray(n, np.float64)
    return n * u / (1 - n * u)


def error_report(got, reference, absval, counts, dtype, alpha, beta_abs=0.0,
                 reference_abs_err=0.0) -> dict:
    """Error of ``got`` against ``reference`` (an FP64 or long-double oracle
    value), and the largest ratio to the stated bound
        |y - y_ref| <= gamma_{n+2}(|alpha| sum|a x| + |beta y0|) + tiny
    (plus ``reference_abs_err``, the reference's own error bound, when the
    reference is not exact).  ``max_ratio_to_bound`` <= 1 means within."""
    # the difference in long double, so a long-double reference is not
    # rounded to FP64 before it is compared
    err = np.abs(np.asarray(got, np.longdouble) -
                 np.asarray(reference, np.longdouble)).astype(np.float64)
    ref = np.asarray(reference, np.float64)
    bound = gamma(np.asarray(counts) + 2, dtype) * (
        abs(alpha) * np.asarray(absval, np.float64) + beta_abs)
    bound = bound + reference_abs_err + np.finfo(dtype).tiny
    scale = np.maximum(np.abs(ref), np.finfo(np.float64).tiny)
    return {"max_abs": float(err.max()) if err.size else 0.0,
            "max_rel": float((err / scale).max()) if err.size else 0.0,
            "max_ratio_to_bound": float((err / bound).max()) if err.size else 0.0,
            "outputs": int(err.size)}
