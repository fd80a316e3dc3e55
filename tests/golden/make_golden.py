"""Generate tests/golden/*.npz from the reference's OWN serial Sparse BLAS.

Run in a checkout where the reference sources are present (they are compiled
into oracle/_ref/libasc_ref.so by oracle/build_oracle.py).  The fixtures pin:

* ``known_answers.npz`` - the known-answer cases of the reference's tests,
  re-run through the reference itself:
    - tests/sparse/blas_test.cc:165-219 (compat SpMV, strided output with
      untouched holes; alpha=2, beta=-0.5 and alpha=1, beta=0),
    - tests/sparse/blas_test.cc:221-242 (row {1e20, 1, -1e20} sums to 0.0f in
      stored order),
    - tests/sparse/blas_test.cc:244-296 (zero columns: y = beta*y),
    - tests/sparse_cuda/sparse_cuda_test.cc:239-352 (4x5 strided SpMV,
      expected {-9,-26,7,-24} and, with beta = 0, {-2,-8,11,-2}),
    - tests/sparse_cuda/sparse_cuda_test.cc:354-433 (2x2 unit stride, {15,29}),
    - tests/sparse/standard_blas_test.cc:177-345 (standard SpMV/SpMM on the
      real part of the 2x2 matrix, CSR none / transpose, CSC, row- and
      column-major B).
* ``random_cases.npz`` - seeded random CSR/CSC matrices, vectors and dense
  right-hand sides with the reference's outputs for compat SpMV, standard SpMV
  (none, transpose) and standard SpMM, FP32 and FP64, unit and non-unit
  strides, empty rows.
* ``laplacian.npz`` - the 5-point Laplacian on a 316 x 316 grid
  (alpha = 1, beta = 0.5, x and y uniform[-1, 1] from seed 0): SHA-256 of the
  reference's output bytes and a strided sample of the output.
* ``conversions.npz`` - the reference's CSR -> CSC, CSC -> CSR and
  coordinate -> CSR / CSC conversions (compressed.h:1676-1780) of the
  conversion test's 3 x 4 matrix (tests/sparse/compressed_conversion_test.cc:
  28-36) and of seeded random matrices with empty rows and columns.
* ``complex_cases.npz`` - complex (Z and C) standard SpMV / SpMM of the
  reference: the complex 2 x 2 known-answer matrix of
  tests/sparse/standard_blas_test.cc:177-345 (CSR none, conjugate transpose,
  CSC none; row-major SpMM, column-major conjugate-transposed CSC SpMM) and a
  seeded random 300 x 220 matrix for every op.
* ``level1_cases.npz`` - the reference's dot (plain and conjugated), axpy,
  gather, gather-zero and scatter on the indexed vector of
  tests/sparse/standard_blas_test.cc:69-173 and on a seeded random one, for
  FP64, FP32, Z and C.
* ``trsv_cases.npz`` - triangular solves: the reference tests' 2 x 2 and 1 x 1
  cases and seeded random 48 x 48 triangular matrices for every triangle,
  diagonal, op and right-hand-side shape, FP64/FP32/Z/C.

Usage:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from asc_cpp_b200 import synthetic  # noqa: E402
from oracle import (CSC, CSR, COL_MAJOR, OP_CONJ_TRANSPOSE, OP_NONE, OP_TRANSPOSE,  # noqa: E402
                    ROW_MAJOR, Reference, build_oracle)


def _check(code: int) -> None:
    if code != 0:
        raise RuntimeError(f"reference returned ErrorCode {code}")


def known_answers(ref: Reference) -> dict[str, np.ndarray]:
    out: dict[str, np.ndarray] = {}
    # blas_test.cc:123-125 matrix, 3x4
    ptr = np.array([0, 2, 4, 5], np.int64)
    idx = np.array([1, 3, 0, 2, 1], np.int64)
    for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
        val = np.array([2, -1, 4, 5, 3], dt)
        x = np.array([2, -1, 3, 4], dt)
        y = np.array([7, -90, 11, -91, 13, -92], dt)
        _check(ref.compat_spmv(3, 4, ptr, idx, val, 2.0, x, -0.5, y, 1, 2))
        out[f"blas_compat_a2_bm05_{tag}"] = y.copy()
        y2 = np.array([np.nan, -90, np.nan, -91, np.nan, -92], dt)
        _check(ref.compat_spmv(3, 4, ptr, idx, val, 1.0, x, 0.0, y2, 1, 2))
        out[f"blas_compat_a1_b0_{tag}"] = y2.copy()
        # zero columns: 3 rows, 0 columns, alpha 7, beta 2
        yz = np.array([2, -3, 4], dt)
        _check(ref.compat_spmv(3, 0, np.zeros(4, np.int64), np.zeros(0, np.int64),
                               np.zeros(0, dt), 7.0, np.zeros(0, dt), 2.0, yz, 1, 1))
        out[f"blas_zero_columns_{tag}"] = yz.copy()
        # empty 3x4 with NaN output, beta = 0
        ye = np.full(3, np.nan, dt)
        _check(ref.compat_spmv(3, 4, np.zeros(4, np.int64), np.zeros(0, np.int64),
                               np.zeros(0, dt), 1.0, np.zeros(4, dt), 0.0, ye, 1, 1))
        out[f"blas_empty_{tag}"] = ye.copy()
    # blas_test.cc:221-242 order test (float)
    yo = np.array([-1.0], np.float32)
    _check(ref.compat_spmv(1, 3, np.array([0, 3], np.int64), np.array([0, 1, 2], np.int64),
                           np.array([1e20, 1, -1e20], np.float32), 1.0,
                           np.ones(3, np.float32), 0.0, yo, 1, 1))
    out["blas_order_f32"] = yo.copy()
    # sparse_cuda_test.cc:239-352 (4x5, x stride 2, y stride 3)
    ptr = np.array([0, 2, 3, 6, 8], np.int64)
    idx = np.array([0, 3, 1, 0, 2, 4, 1, 4], np.int64)
    for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
        val = np.array([2, -1, 4, 7, 3, 5, -2, 6], dt)
        pad = 91
        x = np.array([1, pad, -2, pad, 3, pad, 4, pad, -1], dt)
        y = np.array([10, pad, pad, 20, pad, pad, 30, pad, pad, 40], dt)
        _check(ref.compat_spmv(4, 5, ptr, idx, val, 2.0, x, -0.5, y, 2, 3))
        out[f"cuda_strided_{tag}"] = y.copy()
        yn = np.full(10, np.nan, dt)
        _check(ref.compat_spmv(4, 5, ptr, idx, val, 1.0, x, 0.0, yn, 2, 3))
        out[f"cuda_strided_beta0_{tag}"] = yn.copy()
        # sparse_cuda_test.cc:354-433
        yu = np.array([1, 1], dt)
        _check(ref.compat_spmv(2, 2, np.array([0, 1, 2], np.int64), np.array([0, 1], np.int64),
                               np.array([2, 3], dt), 2.0, np.array([4, 5], dt), -1.0, yu, 1, 1))
        out[f"cuda_unit_{tag}"] = yu.copy()
    # standard_blas_test.cc:177-345 (real parts of its 2x2 matrix)
    ptr = np.array([0, 1, 3], np.int64)
    idx = np.array([0, 0, 1], np.int64)
    cptr = np.array([0, 2, 3], np.int64)
    cidx = np.array([0, 1, 1], np.int64)
    for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
        val = np.array([2.0, 1.0, 3.0], dt)
        x = np.array([1.0, -1.0], dt)
        for op, name in ((OP_NONE, "none"), (OP_TRANSPOSE, "transpose")):
            y = np.zeros(2, dt)
            _check(ref.standard_spmv(CSR, op, 2, 2, ptr, idx, val, 1.0, x, y))
            out[f"std_spmv_csr_{name}_{tag}"] = y.copy()
            y = np.zeros(2, dt)
            _check(ref.standard_spmv(CSC, op, 2, 2, cptr, cidx, val, 1.0, x, y))
            out[f"std_spmv_csc_{name}_{tag}"] = y.copy()
        b = np.array([1.0, 2.0, 3.0, 4.0], dt)
        c = np.zeros(4, dt)
        _check(ref.standard_spmm(CSR, OP_NONE, 2, 2, ptr, idx, val, 1.0, b, 2, 2, ROW_MAJOR, 2,
                                 c, 2, 2, ROW_MAJOR, 2))
        out[f"std_spmm_row_{tag}"] = c.copy()
        b = np.array([1.0, 3.0, 2.0, 4.0], dt)
        c = np.zeros(4, dt)
        _check(ref.standard_spmm(CSC, OP_TRANSPOSE, 2, 2, cptr, cidx, val, 1.0, b, 2, 2,
                                 COL_MAJOR, 2, c, 2, 2, COL_MAJOR, 2))
        out[f"std_spmm_csc_col_t_{tag}"] = c.copy()
    return out


def random_cases(ref: Reference) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(20240611)
    out: dict[str, np.ndarray] = {}
    case = 0
    for dt in (np.float64, np.float32):
        for rows, cols, max_len, empty in ((1, 1, 1, 0.0), (7, 5, 5, 0.3),
                                           (64, 48, 20, 0.1), (200, 300, 40, 0.2),
                                           (513, 129, 70, 0.05)):
            a = synthetic.random_csr(rng, rows, cols, max_len, dt, empty)
            x = rng.uniform(-1, 1, cols).astype(dt)
            xt = rng.uniform(-1, 1, rows).astype(dt)
            y0 = rng.uniform(-1, 1, rows).astype(dt)
            yt0 = rng.uniform(-1, 1, cols).astype(dt)
            alpha, beta = float(rng.choice([1.0, -0.75, 2.5])), float(rng.choice([0.0, 0.5, -1.25]))
            p = f"c{case}_"
            out[p + "shape"] = np.array([rows, cols], np.int64)
            out[p + "ptr"], out[p + "idx"], out[p + "val"] = a.ptr, a.idx, a.val
            out[p + "x"], out[p + "xt"], out[p + "y0"], out[p + "yt0"] = x, xt, y0, yt0
            out[p + "ab"] = np.array([alpha, beta])
            y = y0.copy()
            _check(ref.compat_spmv(rows, cols, a.ptr, a.idx, a.val, alpha, x, beta, y))
            out[p + "compat"] = y
            y = y0.copy()
            _check(ref.standard_spmv(CSR, OP_NONE, rows, cols, a.ptr, a.idx, a.val, alpha, x, y))
            out[p + "std_none"] = y
            y = yt0.copy()
            _check(ref.standard_spmv(CSR, OP_TRANSPOSE, rows, cols, a.ptr, a.idx, a.val, alpha,
                                     xt, y))
            out[p + "std_t"] = y
            k = int(rng.choice([1, 3, 8, 33]))
            b = rng.uniform(-1, 1, cols * k).astype(dt)
            c = rng.uniform(-1, 1, rows * k).astype(dt)
            out[p + "b"], out[p + "c0"] = b, c.copy()
            _check(ref.standard_spmm(CSR, OP_NONE, rows, cols, a.ptr, a.idx, a.val, alpha, b,
                                     cols, k, ROW_MAJOR, k, c, rows, k, ROW_MAJOR, k))
            out[p + "spmm"] = c
            case += 1
    out["count"] = np.array([case])
    return out


def laplacian(ref: Reference) -> dict[str, np.ndarray]:
    a = synthetic.laplacian_2d(316)
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, a.cols)
    y = rng.uniform(-1, 1, a.rows)
    _check(ref.compat_spmv(a.rows, a.cols, a.ptr, a.idx, a.val, 1.0, x, 0.5, y))
    return {"sha256": np.frombuffer(hashlib.sha256(y.tobytes()).digest(), np.uint8),
            "sample_index": np.arange(0, a.rows, 997, dtype=np.int64),
            "sample": y[::997].copy()}


def conversions(ref: Reference) -> dict[str, np.ndarray]:
    """Reference conversions (ConvertToCsc / ConvertToCsr, compressed.h:
    1676-1780) of the conversion test's 3x4 matrix (compressed_conversion_
    test.cc:28-36) and of seeded random matrices with empty rows and columns."""
    out: dict[str, np.ndarray] = {}
    ptr = np.array([0, 2, 4, 5], np.int64)
    idx = np.array([1, 3, 0, 2, 1], np.int64)
    val = np.array([2.0, -1.0, 4.0, 5.0, 3.0])
    coords = np.array([0, 1, 0, 3, 1, 0, 1, 2, 2, 1], np.int64)
    cases = {"ka": (3, 4, ptr, idx, val, coords)}
    rng = np.random.default_rng(21)
    for name, (r, c, m) in {"r1": (60, 45, 12), "r2": (1, 300, 40), "r3": (300, 1, 1),
                            "r4": (200, 700, 9)}.items():
        a = synthetic.random_csr(rng, r, c, m, np.float64, 0.2)
        rows_of = np.repeat(np.arange(r, dtype=np.int64), np.diff(a.ptr))
        co = np.stack([rows_of, a.idx], axis=1).reshape(-1)
        cases[name] = (r, c, a.ptr, a.idx, a.val, co)
    for name, (r, c, p_, i_, v_, co) in cases.items():
        out[f"{name}_shape"] = np.array([r, c], np.int64)
        out[f"{name}_csr_ptr"], out[f"{name}_csr_idx"], out[f"{name}_csr_val"] = p_, i_, v_
        out[f"{name}_coo"] = co
        o, i, v = ref.convert_compressed(1, r, c, p_, i_, v_)
        out[f"{name}_csc_ptr"], out[f"{name}_csc_idx"], out[f"{name}_csc_val"] = o, i, v
        back = ref.convert_compressed(0, r, c, o, i, v)
        for k, arr in zip(("ptr", "idx", "val"), back):
            out[f"{name}_csc_to_csr_{k}"] = arr
        for fmt, to_csc in (("csr", 0), ("csc", 1)):
            o2, i2, v2 = ref.convert_coordinates(to_csc, r, c, co, v_)
            out[f"{name}_coo_to_{fmt}_ptr"] = o2
            out[f"{name}_coo_to_{fmt}_idx"] = i2
            out[f"{name}_coo_to_{fmt}_val"] = v2
    return out


def complex_cases(ref: Reference) -> dict[str, np.ndarray]:
    """The reference's complex standard SpMV / SpMM (blas.h:1607-1750 with
    std::complex elements): the complex 2 x 2 known-answer matrix of
    standard_blas_test.cc:177-345 and seeded random complex matrices."""
    out: dict[str, np.ndarray] = {}
    for dt, tag in ((np.complex128, "z"), (np.complex64, "c")):
        ptr = np.array([0, 1, 3], np.int64)
        idx = np.array([0, 0, 1], np.int64)
        val = np.array([2 + 1j, 1 - 1j, 3 + 0.5j], dt)
        x = np.array([1 + 2j, -1 + 1j], dt)
        for name, fmt, op in (("csr_none", CSR, OP_NONE), ("csr_conjt", CSR, 2)):
            y = np.zeros(2, dt)
            _check(ref.standard_spmv(fmt, op, 2, 2, ptr, idx, val, 1.0, x, y))
            out[f"ka_spmv_{name}_{tag}"] = y
        cptr = np.array([0, 2, 3], np.int64)
        cidx = np.array([0, 1, 1], np.int64)
        y = np.zeros(2, dt)
        _check(ref.standard_spmv(CSC, OP_NONE, 2, 2, cptr, cidx, val, 1.0, x, y))
        out[f"ka_spmv_csc_none_{tag}"] = y
        b = np.array([1, 2, 3, 4], dt)
        c = np.zeros(4, dt)
        _check(ref.standard_spmm(CSR, OP_NONE, 2, 2, ptr, idx, val, 1.0, b, 2, 2, ROW_MAJOR, 2,
                                 c, 2, 2, ROW_MAJOR, 2))
        out[f"ka_spmm_row_{tag}"] = c
        b = np.array([1, 3, 2, 4], dt)
        c = np.zeros(4, dt)
        _check(ref.standard_spmm(CSC, 2, 2, 2, cptr, cidx, val, 1.0, b, 2, 2, COL_MAJOR, 2,
                                 c, 2, 2, COL_MAJOR, 2))
        out[f"ka_spmm_csc_col_conjt_{tag}"] = c
        rng = np.random.default_rng(51 if tag == "z" else 52)
        a = synthetic.random_csr(rng, 300, 220, 25, np.float64, 0.15)
        v = (rng.standard_normal(a.nnz) + 1j * rng.standard_normal(a.nnz)).astype(dt)
        out[f"rand_shape_{tag}"] = np.array([a.rows, a.cols], np.int64)
        out[f"rand_ptr_{tag}"], out[f"rand_idx_{tag}"], out[f"rand_val_{tag}"] = a.ptr, a.idx, v
        alpha = 0.75 - 1.25j
        for op in (OP_NONE, OP_TRANSPOSE, 2):
            nx = a.cols if op == OP_NONE else a.rows
            ny = a.rows if op == OP_NONE else a.cols
            xx = (rng.uniform(-1, 1, nx) + 1j * rng.uniform(-1, 1, nx)).astype(dt)
            yy = (rng.uniform(-1, 1, ny) + 1j * rng.uniform(-1, 1, ny)).astype(dt)
            out[f"rand_x_op{op}_{tag}"], out[f"rand_y0_op{op}_{tag}"] = xx, yy.copy()
            _check(ref.standard_spmv(CSR, op, a.rows, a.cols, a.ptr, a.idx, v, alpha, xx, yy))
            out[f"rand_y_op{op}_{tag}"] = yy
            k = 5
            bb = (rng.uniform(-1, 1, (nx, k)) + 1j * rng.uniform(-1, 1, (nx, k))).astype(dt)
            cc = (rng.uniform(-1, 1, (ny, k)) + 1j * rng.uniform(-1, 1, (ny, k))).astype(dt)
            out[f"rand_b_op{op}_{tag}"], out[f"rand_c0_op{op}_{tag}"] = bb, cc.copy()
            _check(ref.standard_spmm(CSR, op, a.rows, a.cols, a.ptr, a.idx, v, alpha, bb, nx, k,
                                     ROW_MAJOR, k, cc, ny, k, ROW_MAJOR, k))
            out[f"rand_c_op{op}_{tag}"] = cc
    return out


def level1_cases(ref: Reference) -> dict[str, np.ndarray]:
    """The reference's Level-1 operations (blas.h:1340-1600) on the values of
    standard_blas_test.cc:69-173 (indices {0, 2}, dense length 3) and on a
    seeded random indexed vector, for all four element kinds and every op."""
    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(61)
    for dt, tag in ((np.float64, "f64"), (np.float32, "f32"), (np.complex128, "z"),
                    (np.complex64, "c")):
        cplx = np.iscomplexobj(dt(0))
        ka_idx = np.array([0, 2], np.int64)
        ka_val = np.array([1 + 2j, -2 + 1j] if cplx else [1.0, -2.0], dt)
        ka_x = np.array([3 - 1j, 9 + 4j, 2 + 3j] if cplx else [3.0, 9.0, 2.0], dt)
        n = 4000
        r_idx = np.sort(rng.choice(n, 1500, replace=False)).astype(np.int64)
        r_val = (rng.standard_normal(1500) + (1j * rng.standard_normal(1500) if cplx else 0)).astype(dt)
        r_x = (rng.standard_normal(n) + (1j * rng.standard_normal(n) if cplx else 0)).astype(dt)
        alpha = (0.75 - 1.5j) if cplx else 2.0
        for name, (idx, val, x) in (("ka", (ka_idx, ka_val, ka_x)), ("rand", (r_idx, r_val, r_x))):
            out[f"{name}_idx_{tag}"], out[f"{name}_val_{tag}"], out[f"{name}_x_{tag}"] = idx, val, x
            for op in range(5):
                for conj in ((0, 1) if op == 0 else (0,)):
                    v, xx, r = ref.level1(op, conj, idx, val, alpha, x)
                    key = f"{name}_op{op}_conj{conj}_{tag}"
                    out[key + "_val"], out[key + "_x"] = v, xx
                    out[key + "_res"] = np.array([r], dt)
    return out


TRSV_TAGS = (("f64", np.float64), ("f32", np.float32), ("z", np.complex128),
             ("c", np.complex64))
TRSV_SHAPES = ((ROW_MAJOR, 1), (ROW_MAJOR, 3), (COL_MAJOR, 3))


def trsv_cases(ref: Reference) -> dict[str, np.ndarray]:
    """The reference's triangular solves (blas.h:1774-1910): the cases of
    tests/sparse/standard_blas_test.cc:336-420 and
    tests/sparse_cuda/standard_blas_cuda_test.cc:542-680 (the 2 x 2 lower
    matrix with values 2+1i, 1-1i, 3+0.5i solved for (2, -1), its conjugate
    transpose, two right-hand sides, alpha = 0 over NaN values, and the 1 x 1
    complex matrix of magnitude 1e200 / 1e30 divided by itself), then seeded
    random 48 x 48 triangular matrices for every triangle, diagonal, op and
    right-hand-side shape (``rand_<tag>_<triangle><diagonal><op>_<shape>``)."""
    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(67)
    for tag, dt in TRSV_TAGS:
        cplx = np.iscomplexobj(dt(0))
        v = np.array([2 + 1j, 1 - 1j, 3 + 0.5j] if cplx else [2.0, 1.0, 3.0], dt)
        ptr = np.array([0, 1, 3], np.int64)
        idx = np.array([0, 0, 1], np.int64)
        two, m1, one, three = dt(2), dt(-1), dt(1), dt(3)
        cases = {
            "vec": (OP_NONE, np.array([v[0] * two, v[1] * two + v[2] * m1], dt), 1),
            "ct": (OP_CONJ_TRANSPOSE,
                   np.array([np.conj(v[0]) * two - np.conj(v[1]), -np.conj(v[2])], dt), 1),
            "multi": (OP_NONE, np.array([v[0] * two, v[0] * one, v[1] * two + v[2] * m1,
                                         v[1] * one + v[2] * three], dt), 2),
        }
        for name, (op, b, k) in cases.items():
            rc, x = ref.triangular_solve(op, 1, 0, 2, ptr, idx, v, 1.0, b, ROW_MAJOR, k, k)
            _check(rc)
            out[f"ka_{name}_{tag}_b"], out[f"ka_{name}_{tag}_x"] = b, x
        out[f"ka_{tag}_val"] = v
        nan = dt(complex(np.nan, np.nan)) if cplx else dt(np.nan)
        zv = np.array([2, nan, 3], dt)
        rc, x = ref.triangular_solve(OP_NONE, 1, 0, 2, ptr, idx, zv, 0.0,
                                     np.array([4, 5], dt), ROW_MAJOR, 1, 1)
        _check(rc)
        out[f"ka_zero_{tag}_val"], out[f"ka_zero_{tag}_x"] = zv, x
        if cplx:
            big = 1e30 if dt == np.complex64 else 1e200
            lv = np.array([complex(big, big)], dt)
            rc, x = ref.triangular_solve(OP_NONE, 1, 0, 1, np.array([0, 1], np.int64),
                                         np.array([0], np.int64), lv, 1.0, lv, ROW_MAJOR, 1, 1)
            _check(rc)
            out[f"ka_large_{tag}_val"], out[f"ka_large_{tag}_x"] = lv, x
        for triangle in (0, 1):
            for diagonal in (0, 1):
                m = synthetic.triangular(rng, 48, lower=triangle == 1, near=3, far=2,
                                         span=8, dtype=dt)
                for op in (OP_NONE, OP_TRANSPOSE, OP_CONJ_TRANSPOSE):
                    for s, (layout, k) in enumerate(TRSV_SHAPES):
                        b = synthetic._values(rng, 48 * k, dt)
                        alpha = (0.5 - 1.25j) if cplx else -1.5
                        rc, x = ref.triangular_solve(op, triangle, diagonal, 48, m.ptr, m.idx,
                                                     m.val, alpha, b, layout, None, k)
                        _check(rc)
                        key = f"rand_{tag}_{triangle}{diagonal}{op}_{s}"
                        out[key + "_b"], out[key + "_x"] = b, x
                out[f"rand_{tag}_{triangle}{diagonal}_ptr"] = m.ptr
                out[f"rand_{tag}_{triangle}{diagonal}_idx"] = m.idx
                out[f"rand_{tag}_{triangle}{diagonal}_val"] = m.val
    return out


def main() -> None:
    build_oracle.build_reference()
    ref = Reference()
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **known_answers(ref))
    np.savez_compressed(os.path.join(HERE, "random_cases.npz"), **random_cases(ref))
    np.savez_compressed(os.path.join(HERE, "laplacian.npz"), **laplacian(ref))
    np.savez_compressed(os.path.join(HERE, "conversions.npz"), **conversions(ref))
    np.savez_compressed(os.path.join(HERE, "complex_cases.npz"), **complex_cases(ref))
    np.savez_compressed(os.path.join(HERE, "level1_cases.npz"), **level1_cases(ref))
    np.savez_compressed(os.path.join(HERE, "trsv_cases.npz"), **trsv_cases(ref))
    for f in ("known_answers.npz", "random_cases.npz", "laplacian.npz", "conversions.npz",
              "complex_cases.npz", "level1_cases.npz", "trsv_cases.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
