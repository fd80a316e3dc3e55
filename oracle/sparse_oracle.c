/*
 * CPU oracle for the Sparse BLAS hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's serial algorithms, used by tests/,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product path never links, loads or calls this file.
 *
 * Parity of this restatement is pinned two ways (tests/test_oracle.py):
 *   1. bit-exact agreement with oracle/_ref/libasc_ref.so, the reference's own
 *      sources compiled unchanged, on seeded random inputs, and
 *   2. the known-answer vectors of the reference's tests, stored as fixtures
 *      under tests/golden/ together with the script that generated them.
 *
 * Floating point: compiled with -O2 -ffp-contract=off and no -march flag, the
 * same as the reference's x86-64 build, so every * and + rounds separately and
 * no fused multiply-add appears.
 *
 * Layout conventions (the reference's, include/asc/core/types.h:35,62):
 *   CSR: ptr[rows+1], idx[nnz] (column per entry), val[nnz]; int64 indices.
 *   CSC: ptr[cols+1], idx[nnz] (row per entry),    val[nnz].
 *   Vectors: logical element i lives at x[i * inc]; inc may be negative, in
 *   which case x points at logical element 0 (include/asc/sparse/blas.h:1277).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { ORACLE_CSR = 1, ORACLE_CSC = 2 };
enum { ORACLE_OP_NONE = 0, ORACLE_OP_TRANSPOSE = 1, ORACLE_OP_CONJ_TRANSPOSE = 2 };
enum { ORACLE_COL_MAJOR = 0, ORACLE_ROW_MAJOR = 1 };

/* ------------------------------------------------------------------------- */
/* Compat SpMV y = alpha * (sum_k v_k x_{c_k}) + beta * y.
 * Restates SpmvReferenceImpl, src/sparse/reference_blas.cc:9-41:
 *   product starts at Element{} (+0.0) and accumulates value * x[col] in
 *   stored order; result = alpha * product; if beta != 0 then
 *   result += beta * y_old (beta == 0 never reads y); write result.        */
#define ORACLE_COMPAT(SUFFIX, T)                                               \
  void oracle_compat_spmv_##SUFFIX(int64_t rows, const int64_t* ptr,           \
                                   const int64_t* idx, const T* val, T alpha,  \
                                   const T* x, int64_t incx, T beta, T* y,     \
                                   int64_t incy) {                             \
    for (int64_t r = 0; r < rows; ++r) {                                       \
      T product = (T)0;                                                        \
      for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) {                          \
        product += val[p] * x[idx[p] * incx];                                  \
      }                                                                        \
      T result = alpha * product;                                              \
      if (beta != (T)0) {                                                      \
        result += beta * y[r * incy];                                          \
      }                                                                        \
      y[r * incy] = result;                                                    \
    }                                                                          \
  }
ORACLE_COMPAT(f64, double)
ORACLE_COMPAT(f32, float)

/* ------------------------------------------------------------------------- */
/* Standard SpMV y += alpha * op(A) * x.
 * Restates asc::Spmv, include/asc/sparse/blas.h:1607-1667 with ForEachStored
 * (:1241-1256): alpha == 0 returns without touching y; otherwise the stored
 * entries are visited outer index ascending, then stored position ascending,
 * and each does y[out] += alpha * value * x[in] -- evaluated left to right,
 * i.e. (alpha * value) * x[in], then added to y[out].  For CSR outer = row,
 * for CSC outer = column; op != none swaps out and in.  Real types only, so
 * the conjugate transpose equals the transpose.                             */
#define ORACLE_STANDARD_SPMV(SUFFIX, T)                                        \
  void oracle_standard_spmv_##SUFFIX(int format, int op, int64_t rows,         \
                                     int64_t cols, const int64_t* ptr,         \
                                     const int64_t* idx, const T* val,         \
                                     T alpha, const T* x, int64_t incx, T* y,  \
                                     int64_t incy) {                           \
    if (alpha == (T)0) return;                                                 \
    const int64_t outer_extent = format == ORACLE_CSC ? cols : rows;           \
    for (int64_t o = 0; o < outer_extent; ++o) {                               \
      for (int64_t p = ptr[o]; p < ptr[o + 1]; ++p) {                         \
        int64_t row = format == ORACLE_CSC ? idx[p] : o;                       \
        int64_t col = format == ORACLE_CSC ? o : idx[p];                       \
        int64_t out = row, in = col;                                           \
        if (op != ORACLE_OP_NONE) {                                            \
          out = col;                                                           \
          in = row;                                                            \
        }                                                                      \
        y[out * incy] += alpha * val[p] * x[in * incx];                        \
      }                                                                        \
    }                                                                          \
  }
ORACLE_STANDARD_SPMV(f64, double)
ORACLE_STANDARD_SPMV(f32, float)

/* ------------------------------------------------------------------------- */
/* Standard SpMM C += alpha * op(A) * B.
 * Restates asc::Spmm, include/asc/sparse/blas.h:1692-1750: same entry order as
 * SpMV, with an inner loop over the right-hand sides j = 0..ncols-1 doing
 * C(out, j) += alpha * value * B(in, j).  Element (r, c) of a dense matrix is
 * at r*ld + c (row major) or c*ld + r (column major), blas.h:1033-1038.     */
static inline int64_t dense_at(int layout, int64_t ld, int64_t r, int64_t c) {
  return layout == ORACLE_ROW_MAJOR ? r * ld + c : c * ld + r;
}
#define ORACLE_STANDARD_SPMM(SUFFIX, T)                                        \
  void oracle_standard_spmm_##SUFFIX(                                          \
      int format, int op, int64_t rows, int64_t cols, const int64_t* ptr,      \
      const int64_t* idx, const T* val, T alpha, const T* b, int b_layout,     \
      int64_t ldb, T* c, int c_layout, int64_t ldc, int64_t ncols) {           \
    if (alpha == (T)0) return;                                                 \
    const int64_t outer_extent = format == ORACLE_CSC ? cols : rows;           \
    for (int64_t o = 0; o < outer_extent; ++o) {                               \
      for (int64_t p = ptr[o]; p < ptr[o + 1]; ++p) {                         \
        int64_t row = format == ORACLE_CSC ? idx[p] : o;                       \
        int64_t col = format == ORACLE_CSC ? o : idx[p];                       \
        int64_t out = row, in = col;                                           \
        if (op != ORACLE_OP_NONE) {                                            \
          out = col;                                                           \
          in = row;                                                            \
        }                                                                      \
        for (int64_t j = 0; j < ncols; ++j) {                                  \
          c[dense_at(c_layout, ldc, out, j)] +=                                \
              alpha * val[p] * b[dense_at(b_layout, ldb, in, j)];              \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }
ORACLE_STANDARD_SPMM(f64, double)
ORACLE_STANDARD_SPMM(f32, float)

/* ------------------------------------------------------------------------- */
/* Complex standard SpMV / SpMM: the same loops over interleaved (re, im)
 * storage, the layout of std::complex<T> (two T, real first).  Each entry
 * does out += (alpha * v') * in with v' = conj(v) for the conjugate
 * transpose (blas.h:1653-1665, 1739-1748; MaybeConjugate).  A complex product
 * (a, b) * (c, d) is (ac - bd, ad + bc) with every product and sum rounded
 * separately and a sum is component-wise: the value std::complex<T> gives
 * under GCC without -march (no contraction) whenever the result is not
 * NaN + NaN i -- only then does C99 Annex G's recovery (__muldc3) differ,
 * so the oracle, like the tests, covers finite data.                       */
#define ORACLE_COMPLEX(SUFFIX, T)                                              \
  static inline void cmul_##SUFFIX(T ar, T ai, T br, T bi, T* r, T* i) {       \
    const T rr = ar * br;                                                      \
    const T ii = ai * bi;                                                      \
    const T ri = ar * bi;                                                      \
    const T ir = ai * br;                                                      \
    *r = rr - ii;                                                              \
    *i = ri + ir;                                                              \
  }                                                                            \
  void oracle_complex_spmv_##SUFFIX(int format, int op, int64_t rows,          \
                                    int64_t cols, const int64_t* ptr,          \
                                    const int64_t* idx, const T* val, T al_r,  \
                                    T al_i, const T* x, int64_t incx, T* y,    \
                                    int64_t incy) {                            \
    if (al_r == (T)0 && al_i == (T)0) return;                                  \
    const int64_t outer_extent = format == ORACLE_CSC ? cols : rows;           \
    for (int64_t o = 0; o < outer_extent; ++o) {                               \
      for (int64_t p = ptr[o]; p < ptr[o + 1]; ++p) {                         \
        int64_t row = format == ORACLE_CSC ? idx[p] : o;                       \
        int64_t col = format == ORACLE_CSC ? o : idx[p];                       \
        int64_t out = row, in = col;                                           \
        T vr = val[2 * p], vi = val[2 * p + 1];                                \
        if (op != ORACLE_OP_NONE) {                                            \
          out = col;                                                           \
          in = row;                                                            \
          if (op == ORACLE_OP_CONJ_TRANSPOSE) vi = -vi;                        \
        }                                                                      \
        T tr, ti, pr, pi;                                                      \
        cmul_##SUFFIX(al_r, al_i, vr, vi, &tr, &ti);                           \
        cmul_##SUFFIX(tr, ti, x[2 * in * incx], x[2 * in * incx + 1], &pr,     \
                      &pi);                                                    \
        y[2 * out * incy] += pr;                                               \
        y[2 * out * incy + 1] += pi;                                           \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  void oracle_complex_spmm_##SUFFIX(                                           \
      int format, int op, int64_t rows, int64_t cols, const int64_t* ptr,      \
      const int64_t* idx, const T* val, T al_r, T al_i, const T* b,            \
      int b_layout, int64_t ldb, T* c, int c_layout, int64_t ldc,              \
      int64_t ncols) {                                                         \
    if (al_r == (T)0 && al_i == (T)0) return;                                  \
    const int64_t outer_extent = format == ORACLE_CSC ? cols : rows;           \
    for (int64_t o = 0; o < outer_extent; ++o) {                               \
      for (int64_t p = ptr[o]; p < ptr[o + 1]; ++p) {                         \
        int64_t row = format == ORACLE_CSC ? idx[p] : o;                       \
        int64_t col = format == ORACLE_CSC ? o : idx[p];                       \
        int64_t out = row, in = col;                                           \
        T vr = val[2 * p], vi = val[2 * p + 1];                                \
        if (op != ORACLE_OP_NONE) {                                            \
          out = col;                                                           \
          in = row;                                                            \
          if (op == ORACLE_OP_CONJ_TRANSPOSE) vi = -vi;                        \
        }                                                                      \
        T tr, ti;                                                              \
        cmul_##SUFFIX(al_r, al_i, vr, vi, &tr, &ti);                           \
        for (int64_t j = 0; j < ncols; ++j) {                                  \
          const int64_t bi = dense_at(b_layout, ldb, in, j);                   \
          const int64_t ci = dense_at(c_layout, ldc, out, j);                  \
          T pr, pi;                                                            \
          cmul_##SUFFIX(tr, ti, b[2 * bi], b[2 * bi + 1], &pr, &pi);           \
          c[2 * ci] += pr;                                                     \
          c[2 * ci + 1] += pi;                                                 \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }
ORACLE_COMPLEX(z, double)
ORACLE_COMPLEX(c, float)

/* ------------------------------------------------------------------------- */
/* Level-1 on an indexed vector (blas.h:1340-1600): op 0 dot (serial, from
 * zero, result += v' * x[i]), 1 axpy (x[i] += alpha * v), 2 gather, 3
 * gather-zero, 4 scatter.  Complex variants work on (re, im) pairs with the
 * products of ORACLE_COMPLEX above.                                        */
#define ORACLE_LEVEL1(SUFFIX, T)                                               \
  void oracle_level1_##SUFFIX(int op, int conj, const int64_t* idx, T* val,    \
                              int64_t nnz, T alpha, T* x, T* result) {         \
    (void)conj;                                                                \
    if (op == 0) {                                                             \
      T sum = (T)0;                                                            \
      for (int64_t q = 0; q < nnz; ++q) sum += val[q] * x[idx[q]];             \
      *result = sum;                                                           \
      return;                                                                  \
    }                                                                          \
    if (op == 1 && alpha == (T)0) return;                                      \
    for (int64_t q = 0; q < nnz; ++q) {                                        \
      T* xi = &x[idx[q]];                                                      \
      if (op == 1) *xi += alpha * val[q];                                      \
      if (op == 2) val[q] = *xi;                                               \
      if (op == 3) { val[q] = *xi; *xi = (T)0; }                               \
      if (op == 4) *xi = val[q];                                               \
    }                                                                          \
  }
ORACLE_LEVEL1(f64, double)
ORACLE_LEVEL1(f32, float)

#define ORACLE_LEVEL1_COMPLEX(SUFFIX, T)                                       \
  void oracle_level1_##SUFFIX(int op, int conj, const int64_t* idx, T* val,    \
                              int64_t nnz, T al_r, T al_i, T* x, T* result) {  \
    if (op == 0) {                                                             \
      T sr = (T)0, si = (T)0;                                                  \
      for (int64_t q = 0; q < nnz; ++q) {                                      \
        T pr, pi;                                                              \
        const T vi = conj ? -val[2 * q + 1] : val[2 * q + 1];                  \
        cmul_##SUFFIX(val[2 * q], vi, x[2 * idx[q]], x[2 * idx[q] + 1], &pr,   \
                      &pi);                                                    \
        sr += pr;                                                              \
        si += pi;                                                              \
      }                                                                        \
      result[0] = sr;                                                          \
      result[1] = si;                                                          \
      return;                                                                  \
    }                                                                          \
    if (op == 1 && al_r == (T)0 && al_i == (T)0) return;                       \
    for (int64_t q = 0; q < nnz; ++q) {                                        \
      T* xi = &x[2 * idx[q]];                                                  \
      if (op == 1) {                                                           \
        T pr, pi;                                                              \
        cmul_##SUFFIX(al_r, al_i, val[2 * q], val[2 * q + 1], &pr, &pi);       \
        xi[0] += pr;                                                           \
        xi[1] += pi;                                                           \
      }                                                                        \
      if (op == 2) { val[2 * q] = xi[0]; val[2 * q + 1] = xi[1]; }             \
      if (op == 3) {                                                           \
        val[2 * q] = xi[0]; val[2 * q + 1] = xi[1]; xi[0] = (T)0; xi[1] = (T)0; \
      }                                                                        \
      if (op == 4) { xi[0] = val[2 * q]; xi[1] = val[2 * q + 1]; }             \
    }                                                                          \
  }
ORACLE_LEVEL1_COMPLEX(z, double)
ORACLE_LEVEL1_COMPLEX(c, float)

/* ------------------------------------------------------------------------- */
/* Extended-precision companions used to state and check error bounds.
 * For each output o of op(A) (CSR, unit-stride vectors) they return
 *   exact[o] ~= sum_k v_k x_k   (long double accumulation of exact products)
 *   absval[o] = sum_k |v_k| |x_k|
 * so that a result r can be checked against |r - exact| <= g * absval.     */
#define ORACLE_EXTENDED(SUFFIX, T)                                             \
  void oracle_csr_extended_##SUFFIX(int op, int64_t rows, int64_t cols,        \
                                    const int64_t* ptr, const int64_t* idx,    \
                                    const T* val, const T* x,                  \
                                    long double* exact, long double* absval) { \
    const int64_t n_out = op == ORACLE_OP_NONE ? rows : cols;                  \
    for (int64_t o = 0; o < n_out; ++o) {                                      \
      exact[o] = 0.0L;                                                         \
      absval[o] = 0.0L;                                                        \
    }                                                                          \
    for (int64_t r = 0; r < rows; ++r) {                                       \
      for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) {                         \
        const int64_t out = op == ORACLE_OP_NONE ? r : idx[p];                 \
        const int64_t in = op == ORACLE_OP_NONE ? idx[p] : r;                  \
        const long double prod = (long double)val[p] * (long double)x[in];     \
        exact[out] += prod;                                                    \
        absval[out] += fabsl(prod);                                            \
      }                                                                        \
    }                                                                          \
  }
ORACLE_EXTENDED(f64, double)
ORACLE_EXTENDED(f32, float)

/* Row lengths of op(A): the n in gamma_n for each output. */
void oracle_output_counts(int op, int64_t rows, int64_t cols,
                          const int64_t* ptr, const int64_t* idx,
                          int64_t* counts) {
  const int64_t n_out = op == ORACLE_OP_NONE ? rows : cols;
  memset(counts, 0, (size_t)n_out * sizeof(int64_t));
  for (int64_t r = 0; r < rows; ++r) {
    if (op == ORACLE_OP_NONE) {
      counts[r] = ptr[r + 1] - ptr[r];
    } else {
      for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) counts[idx[p]] += 1;
    }
  }
}

/* ------------------------------------------------------------------------- */
/* CSR -> CSC (equivalently: the CSR structure of A^T), integer work.
 * Restates the column-major re-compression of
 * CompressedSparseArray::FromCompressed, include/asc/sparse/compressed.h:
 * 1151-1221: entries of each output column appear in increasing source row,
 * which is exactly the order the standard transpose visits them
 * (blas.h:1241-1256).  perm[q] = source position of transposed entry q.     */
void oracle_csr_transpose_structure(int64_t rows, int64_t cols,
                                    const int64_t* ptr, const int64_t* idx,
                                    int64_t* t_ptr, int64_t* t_idx,
                                    int64_t* perm) {
  memset(t_ptr, 0, (size_t)(cols + 1) * sizeof(int64_t));
  const int64_t nnz = ptr[rows];
  for (int64_t p = 0; p < nnz; ++p) t_ptr[idx[p] + 1] += 1;
  for (int64_t c = 0; c < cols; ++c) t_ptr[c + 1] += t_ptr[c];
  int64_t* next = (int64_t*)malloc((size_t)(cols > 0 ? cols : 1) * sizeof(int64_t));
  if (next == NULL) return;
  memcpy(next, t_ptr, (size_t)cols * sizeof(int64_t));
  for (int64_t r = 0; r < rows; ++r) {
    for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) {
      const int64_t q = next[idx[p]]++;
      t_idx[q] = r;
      perm[q] = p;
    }
  }
  free(next);
}

/* ------------------------------------------------------------------------- */
/* Stable bucket sort of n entries by key = keys[e * kstride] in [0, limit):
 * offsets[0..limit] are the bucket starts, perm[q] the source position of the
 * q-th entry in (key, source position) order.  It is the order in which the
 * reference's conversions emit entries: FromCompressed scans every source
 * outer in order for each destination outer (compressed.h:1151-1221) and
 * FromCoordinate scans every coordinate in stored order for each destination
 * outer (compressed.h:1082-1131), so within one destination outer entries
 * keep their source order.  Keys outside [0, limit) are a contract violation
 * and are left out (their perm slots are -1 at the end). */
void oracle_stable_bucket_sort(int64_t n, const int64_t* keys, int64_t kstride,
                               int64_t limit, int64_t* offsets,
                               int64_t* perm) {
  memset(offsets, 0, (size_t)(limit + 1) * sizeof(int64_t));
  for (int64_t e = 0; e < n; ++e) {
    const int64_t k = keys[e * kstride];
    if (k >= 0 && k < limit) offsets[k + 1] += 1;
  }
  for (int64_t k = 0; k < limit; ++k) offsets[k + 1] += offsets[k];
  int64_t* next = (int64_t*)malloc((size_t)(limit > 0 ? limit : 1) * sizeof(int64_t));
  if (next == NULL) return;
  memcpy(next, offsets, (size_t)limit * sizeof(int64_t));
  for (int64_t q = offsets[limit]; q < n; ++q) perm[q] = -1;
  for (int64_t e = 0; e < n; ++e) {
    const int64_t k = keys[e * kstride];
    if (k >= 0 && k < limit) perm[next[k]++] = e;
  }
  free(next);
}

/* ------------------------------------------------------------------------- */
/* Merge-path split of the (row-end, nonzero) merge of a CSR matrix.
 * The merge interleaves list A = ptr[1..rows] (the end offset of each row)
 * with list B = 0, 1, ..., nnz-1 (the nonzero positions), taking a nonzero
 * while its position is below the current row's end.  Diagonal d of the
 * merge grid is split at (i, d - i): i row ends and d - i nonzeros consumed.
 * i is found by binary search as the first candidate in
 * [max(0, d - nnz), min(d, rows)] with A[i] > B[d - i - 1]
 * (Odeh et al., "Merge Path", 2012; applied to CSR SpMV by Merrill and
 * Garland, 2016).  The reference has no counterpart; the GPU partition kernel
 * must reproduce these integers exactly.                                    */
void oracle_merge_path_split(int64_t rows, const int64_t* ptr, int64_t nnz,
                             int64_t diagonal, int64_t* row_out,
                             int64_t* nz_out) {
  int64_t lo = diagonal - nnz > 0 ? diagonal - nnz : 0;
  int64_t hi = diagonal < rows ? diagonal : rows;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (ptr[mid + 1] <= diagonal - mid - 1) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  *row_out = lo;
  *nz_out = diagonal - lo;
}

/* ------------------------------------------------------------------------- */
/* Sparse triangular solve op(A) X = alpha B, X overwriting B (n x k, dense
 * layout/ld as in SpMM), for square CSR A.  Restates SparseTriangularSolve /
 * SparseTriangularSolveMultiple (include/asc/sparse/blas.h:1774-1831,
 * 1856-1910) and the CUDA facet's StandardTriangularSolveKernel
 * (src/sparse/cuda/kernels.cu:349-391):
 *   * alpha == 0: X = 0 (every element, both parts zero for complex);
 *   * M = op(A); M is lower triangular when (op == none and triangle ==
 *     lower) or (op != none and triangle == upper), and rows run 0..n-1 for
 *     lower M, n-1..0 for upper M;
 *   * value = alpha * B(row); then for each column c of the row's strict
 *     triangle in increasing order value -= M(row, c) * X(c); with a non-unit
 *     diagonal value /= M(row, row); X(row) = value.
 * M(row, c) = A(c, row) for transposed ops, conjugated for the conjugate
 * transpose.  The reference loops over every column and subtracts
 * OpValue * X(c) with OpValue = 0 for entries that are not stored; this
 * restatement visits stored entries only, which gives the same result
 * whenever X holds finite values and no running value is a negative zero
 * (a skipped 0 * x can only turn -0 into +0 or make Inf/NaN).  Stored
 * entries outside the strict triangle other than the diagonal are ignored,
 * as the CUDA facet ignores them.  A missing diagonal divides by zero, as
 * the facet's CsrOpValue returns zero for it.
 * Complex division follows the facet's DeviceArithmetic::Divide
 * (kernels.cu:58-72), Smith's method (Smith, CACM 5(8), 1962): with
 * d = dr + i di and |dr| >= |di|, r = di/dr, t = dr + di r,
 * q = ((nr + ni r)/t, (ni - nr r)/t); otherwise r = dr/di, t = di + dr r,
 * q = ((nr r + ni)/t, (ni r - nr)/t).                                       */
enum { ORACLE_UPPER = 0, ORACLE_LOWER = 1 };
enum { ORACLE_NON_UNIT = 0, ORACLE_UNIT = 1 };

/* CSR of M = op(A): the stored arrays for op == none, else the stable
 * transposed structure with values permuted.  Returns 0 on success. */
static int oracle_op_csr(int op, int64_t n, const int64_t* ptr, const int64_t* idx,
                         int64_t** m_ptr, int64_t** m_idx, int64_t** m_perm) {
  const int64_t nnz = ptr[n];
  *m_ptr = (int64_t*)malloc((size_t)(n + 1) * sizeof(int64_t));
  *m_idx = (int64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
  *m_perm = (int64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
  if (*m_ptr == NULL || *m_idx == NULL || *m_perm == NULL) return -1;
  if (op == ORACLE_OP_NONE) {
    memcpy(*m_ptr, ptr, (size_t)(n + 1) * sizeof(int64_t));
    for (int64_t p = 0; p < nnz; ++p) {
      (*m_idx)[p] = idx[p];
      (*m_perm)[p] = p;
    }
    return 0;
  }
  oracle_csr_transpose_structure(n, n, ptr, idx, *m_ptr, *m_idx, *m_perm);
  return 0;
}

#define ORACLE_TRSV(SUFFIX, T)                                                 \
  int oracle_trsv_##SUFFIX(int op, int triangle, int diagonal, int64_t n,      \
                           const int64_t* ptr, const int64_t* idx,             \
                           const T* val, T alpha, T* b, int layout, int64_t ld,\
                           int64_t k) {                                        \
    if (alpha == (T)0) {                                                       \
      for (int64_t j = 0; j < k; ++j)                                          \
        for (int64_t r = 0; r < n; ++r) b[dense_at(layout, ld, r, j)] = (T)0;  \
      return 0;                                                                \
    }                                                                          \
    int64_t *mp, *mi, *mq;                                                     \
    if (oracle_op_csr(op, n, ptr, idx, &mp, &mi, &mq) != 0) return -1;         \
    const int lower = op == ORACLE_OP_NONE ? triangle == ORACLE_LOWER          \
                                           : triangle == ORACLE_UPPER;         \
    for (int64_t j = 0; j < k; ++j) {                                          \
      for (int64_t s = 0; s < n; ++s) {                                        \
        const int64_t row = lower ? s : n - 1 - s;                             \
        T value = alpha * b[dense_at(layout, ld, row, j)];                     \
        T diag = (T)0;                                                         \
        for (int64_t p = mp[row]; p < mp[row + 1]; ++p) {                      \
          const int64_t c = mi[p];                                             \
          if (c == row) diag = val[mq[p]];                                     \
          if ((lower && c >= row) || (!lower && c <= row)) continue;           \
          value -= val[mq[p]] * b[dense_at(layout, ld, c, j)];                 \
        }                                                                      \
        if (diagonal == ORACLE_NON_UNIT) value /= diag;                        \
        b[dense_at(layout, ld, row, j)] = value;                               \
      }                                                                        \
    }                                                                          \
    free(mp);                                                                  \
    free(mi);                                                                  \
    free(mq);                                                                  \
    return 0;                                                                  \
  }
ORACLE_TRSV(f64, double)
ORACLE_TRSV(f32, float)

#define ORACLE_TRSV_COMPLEX(SUFFIX, T)                                         \
  static inline void cdiv_##SUFFIX(T nr, T ni, T dr, T di, T* qr, T* qi) {     \
    const T adr = dr < (T)0 ? -dr : dr;                                        \
    const T adi = di < (T)0 ? -di : di;                                        \
    if (adr >= adi) {                                                          \
      const T ratio = di / dr;                                                 \
      const T den = dr + di * ratio;                                           \
      *qr = (nr + ni * ratio) / den;                                           \
      *qi = (ni - nr * ratio) / den;                                           \
    } else {                                                                   \
      const T ratio = dr / di;                                                 \
      const T den = di + dr * ratio;                                           \
      *qr = (nr * ratio + ni) / den;                                           \
      *qi = (ni * ratio - nr) / den;                                           \
    }                                                                          \
  }                                                                            \
  int oracle_trsv_##SUFFIX(int op, int triangle, int diagonal, int64_t n,      \
                           const int64_t* ptr, const int64_t* idx,             \
                           const T* val, T al_r, T al_i, T* b, int layout,     \
                           int64_t ld, int64_t k) {                            \
    if (al_r == (T)0 && al_i == (T)0) {                                        \
      for (int64_t j = 0; j < k; ++j)                                          \
        for (int64_t r = 0; r < n; ++r) {                                      \
          const int64_t e = dense_at(layout, ld, r, j);                        \
          b[2 * e] = (T)0;                                                     \
          b[2 * e + 1] = (T)0;                                                 \
        }                                                                      \
      return 0;                                                                \
    }                                                                          \
    int64_t *mp, *mi, *mq;                                                     \
    if (oracle_op_csr(op, n, ptr, idx, &mp, &mi, &mq) != 0) return -1;         \
    const int lower = op == ORACLE_OP_NONE ? triangle == ORACLE_LOWER          \
                                           : triangle == ORACLE_UPPER;         \
    const int conj = op == ORACLE_OP_CONJ_TRANSPOSE;                           \
    for (int64_t j = 0; j < k; ++j) {                                          \
      for (int64_t s = 0; s < n; ++s) {                                        \
        const int64_t row = lower ? s : n - 1 - s;                             \
        const int64_t e = dense_at(layout, ld, row, j);                        \
        T vr, vi;                                                              \
        cmul_##SUFFIX(al_r, al_i, b[2 * e], b[2 * e + 1], &vr, &vi);           \
        T dr = (T)0, di = (T)0;                                                \
        for (int64_t p = mp[row]; p < mp[row + 1]; ++p) {                      \
          const int64_t c = mi[p];                                             \
          const T mr = val[2 * mq[p]];                                         \
          const T mi_ = conj ? -val[2 * mq[p] + 1] : val[2 * mq[p] + 1];       \
          if (c == row) {                                                      \
            dr = mr;                                                           \
            di = mi_;                                                          \
          }                                                                    \
          if ((lower && c >= row) || (!lower && c <= row)) continue;           \
          const int64_t xe = dense_at(layout, ld, c, j);                       \
          T pr, pi;                                                            \
          cmul_##SUFFIX(mr, mi_, b[2 * xe], b[2 * xe + 1], &pr, &pi);          \
          vr -= pr;                                                            \
          vi -= pi;                                                            \
        }                                                                      \
        if (diagonal == ORACLE_NON_UNIT) cdiv_##SUFFIX(vr, vi, dr, di, &vr, &vi); \
        b[2 * e] = vr;                                                         \
        b[2 * e + 1] = vi;                                                     \
      }                                                                        \
    }                                                                          \
    free(mp);                                                                  \
    free(mi);                                                                  \
    free(mq);                                                                  \
    return 0;                                                                  \
  }
ORACLE_TRSV_COMPLEX(z, double)
ORACLE_TRSV_COMPLEX(c, float)
