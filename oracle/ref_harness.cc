// Test infrastructure only: a C-ABI harness around the reference's OWN serial
// Sparse BLAS, compiled from the reference sources (never copied into this
// repository) by oracle/build_oracle.py into oracle/_ref/libasc_ref.so.
//
// It is the checker for the hand-written C restatement in oracle/sparse_oracle.c
// and the CPU arm of bench.py.  Nothing on the product path links or loads it.
//
// Entry points call the public reference templates exactly as a caller would:
//   * compat SpMV   asc::Spmv(ctx, alpha, CsrView, x, beta, y)
//                   include/asc/sparse/blas.h:2031-2081 ->
//                   src/sparse/reference_blas.cc:9-41 (SpmvReferenceImpl)
//   * standard SpMV asc::Spmv(ctx, op, alpha, CompressedSparseView, x, y)
//                   include/asc/sparse/blas.h:1607-1667
//   * standard SpMM asc::Spmm(ctx, op, alpha, CompressedSparseView, B, C)
//                   include/asc/sparse/blas.h:1692-1750
//   * triangular    asc::SparseTriangularSolveMultiple (blas.h:1856-1910)
//   * conversions   asc::ConvertToCsr / ConvertToCsc (compressed.h:1676-1780)
//                   -> CompressedSparseArray::FromCompressed (:1151-1221)
//                   and FromCoordinate (:1082-1131)
// Return value: the reference's asc::ErrorCode as an int (0 == kOk).

#include <algorithm>
#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <span>
#include <thread>
#include <vector>

#include "asc/core/execution.h"
#include "asc/core/memory.h"
#include "asc/core/status.h"
#include "asc/core/types.h"
#include "asc/expression/expression.h"
#include "asc/expression/writable.h"
#include "asc/sparse/blas.h"
#include "asc/sparse/compressed.h"
#include "asc/sparse/coordinate.h"

// A strided host vector made visible to the reference's expression protocol.
template <typename T>
struct HarnessVector {
  T* data = nullptr;
  asc::extent_t size = 0;
  asc::stride_t stride = 1;
  std::size_t Bytes() const {
    if (size <= 0) return 0;
    return static_cast<std::size_t>((size - 1) * stride + 1) * sizeof(T);
  }
};

namespace asc {

template <typename T>
struct ExpressionAdapter<::HarnessVector<T>> {
  using value_type = std::remove_const_t<T>;
  static constexpr rank_t rank = 1;
  static constexpr SparsityEffect sparsity_effect =
      SparsityEffect::kStructurePreserving;
  static constexpr ExpressionOperation operation =
      ExpressionOperation::kExternal;
  static constexpr std::array<extent_t, 1> Shape(
      const ::HarnessVector<T>& v) noexcept {
    return {v.size};
  }
  static value_type Read(const ::HarnessVector<T>& v,
                         std::span<const index_t, 1> c) noexcept {
    return v.data[c[0] * v.stride];
  }
  static bool MayAlias(const ::HarnessVector<T>& v, AliasToken token) noexcept {
    if (v.data == nullptr || v.size <= 0 || token.identity() == nullptr) {
      return false;
    }
    const auto begin = reinterpret_cast<std::uintptr_t>(v.data);
    const auto address = reinterpret_cast<std::uintptr_t>(token.identity());
    return address >= begin && address < begin + v.Bytes();
  }
};

template <typename T>
struct ExpressionPlacementAdapter<::HarnessVector<T>> {
  static constexpr MemorySpace Space(const ::HarnessVector<T>&) noexcept {
    return MemorySpace::kHost;
  }
  static ExpressionAliasMetadata Alias(const ::HarnessVector<T>& v) noexcept {
    return ExpressionAliasMetadata(v.data, v.data, v.Bytes());
  }
};

template <typename T>
  requires(!std::is_const_v<T>)
struct WritableExpressionAdapter<::HarnessVector<T>> {
  using value_type = T;
  static constexpr std::array<extent_t, 1> Shape(
      const ::HarnessVector<T>& v) noexcept {
    return {v.size};
  }
  static ExpressionAliasMetadata Alias(const ::HarnessVector<T>& v) noexcept {
    return ExpressionPlacementAdapter<::HarnessVector<T>>::Alias(v);
  }
  static constexpr bool IsUnique(const ::HarnessVector<T>&) noexcept {
    return true;
  }
  static void Write(::HarnessVector<T>& v, std::span<const index_t, 1> c,
                    value_type value) noexcept {
    v.data[c[0] * v.stride] = value;
  }
};

}  // namespace asc

namespace {

int Code(const asc::Status& s) { return static_cast<int>(s.code()); }

template <typename T>
int CompatSpmv(std::int64_t rows, std::int64_t cols, const std::int64_t* ptr,
               const std::int64_t* idx, const T* val, std::int64_t nnz,
               T alpha, const T* x, std::int64_t incx, T beta, T* y,
               std::int64_t incy) {
  const std::array<asc::extent_t, 2> shape{rows, cols};
  auto m = asc::CsrView<const T>::Create(ptr, idx, val, shape, nnz,
                                         asc::MemorySpace::kHost);
  if (!m.ok()) return Code(m.status());
  const HarnessVector<const T> in{x, cols, incx};
  HarnessVector<T> out{y, rows, incy};
  return Code(asc::Spmv(asc::ExecutionContext::Serial(), alpha, *m, in, beta,
                        out));
}

asc::SparseBlasTranspose Op(int op) {
  return static_cast<asc::SparseBlasTranspose>(op);
}

template <typename T>
asc::ConstMemoryView ConstSpan(const T* p, std::size_t count) {
  return {p, count * sizeof(T), asc::MemorySpace::kHost};
}

template <typename T, asc::SparseCompressedFormat F>
int StandardSpmvTyped(int op, std::int64_t rows, std::int64_t cols,
                      const std::int64_t* ptr, const std::int64_t* idx,
                      const T* val, std::int64_t nnz, T alpha, const T* x,
                      std::int64_t nx, std::int64_t incx,
                      std::size_t x_storage, T* y, std::int64_t ny,
                      std::int64_t incy, std::size_t y_storage) {
  const std::array<asc::extent_t, 2> shape{rows, cols};
  auto m = asc::CompressedSparseView<const T, F>::Create(
      ptr, idx, val, shape, nnz, asc::MemorySpace::kHost);
  if (!m.ok()) return Code(m.status());
  // x / y point at logical element 0; for a negative increment the backing
  // storage starts (n-1)*|inc| elements earlier.
  const T* x_base = incx < 0 && nx > 0 ? x + (nx - 1) * incx : x;
  T* y_base = incy < 0 && ny > 0 ? y + (ny - 1) * incy : y;
  auto in = asc::SparseBlasVectorView<const T>::Create(
      x, nx, incx, ConstSpan(x_base, x_storage));
  if (!in.ok()) return Code(in.status());
  auto out = asc::SparseBlasVectorView<T>::Create(
      y, ny, incy,
      asc::MutableMemoryView(y_base, y_storage * sizeof(T),
                             asc::MemorySpace::kHost));
  if (!out.ok()) return Code(out.status());
  return Code(asc::Spmv(asc::ExecutionContext::Serial(), Op(op), alpha, *m,
                        *in, *out));
}

template <typename T, asc::SparseCompressedFormat F>
int StandardSpmmTyped(int op, std::int64_t rows, std::int64_t cols,
                      const std::int64_t* ptr, const std::int64_t* idx,
                      const T* val, std::int64_t nnz, T alpha, const T* b,
                      std::int64_t b_rows, std::int64_t b_cols, int b_layout,
                      std::int64_t ldb, std::size_t b_storage, T* c,
                      std::int64_t c_rows, std::int64_t c_cols, int c_layout,
                      std::int64_t ldc, std::size_t c_storage) {
  const std::array<asc::extent_t, 2> shape{rows, cols};
  auto m = asc::CompressedSparseView<const T, F>::Create(
      ptr, idx, val, shape, nnz, asc::MemorySpace::kHost);
  if (!m.ok()) return Code(m.status());
  auto in = asc::SparseBlasMatrixView<const T>::Create(
      b, b_rows, b_cols, static_cast<asc::SparseBlasLayout>(b_layout), ldb,
      ConstSpan(b, b_storage));
  if (!in.ok()) return Code(in.status());
  auto out = asc::SparseBlasMatrixView<T>::Create(
      c, c_rows, c_cols, static_cast<asc::SparseBlasLayout>(c_layout), ldc,
      asc::MutableMemoryView(c, c_storage * sizeof(T),
                             asc::MemorySpace::kHost));
  if (!out.ok()) return Code(out.status());
  return Code(asc::Spmm(asc::ExecutionContext::Serial(), Op(op), alpha, *m,
                        *in, *out));
}

// Row-block decomposition of one CSR matrix so that several host threads can
// each run the reference's serial compat SpMV on a disjoint block of rows.
// Every row's arithmetic is still the reference's own, unchanged.
template <typename T>
struct Blocks {
  std::int64_t cols = 0;
  std::vector<std::int64_t> row_begin;
  std::vector<std::vector<std::int64_t>> offsets;  // rebased to zero
  std::vector<asc::CsrView<const T>> views;
};

template <typename T>
void* PrepareBlocks(std::int64_t rows, std::int64_t cols,
                    const std::int64_t* ptr, const std::int64_t* idx,
                    const T* val, int nblocks) {
  auto blocks = std::make_unique<Blocks<T>>();
  blocks->cols = cols;
  const std::int64_t nnz = ptr[rows];
  nblocks = std::max(1, nblocks);
  blocks->row_begin.push_back(0);
  for (int b = 1; b < nblocks; ++b) {
    // nnz-balanced split
    const std::int64_t target = nnz * b / nblocks;
    std::int64_t r = std::lower_bound(ptr, ptr + rows + 1, target) - ptr;
    r = std::clamp(r, blocks->row_begin.back(), rows);
    blocks->row_begin.push_back(r);
  }
  blocks->row_begin.push_back(rows);
  for (int b = 0; b < nblocks; ++b) {
    const std::int64_t r0 = blocks->row_begin[b];
    const std::int64_t r1 = blocks->row_begin[b + 1];
    std::vector<std::int64_t> off(static_cast<std::size_t>(r1 - r0 + 1));
    for (std::int64_t r = r0; r <= r1; ++r) off[r - r0] = ptr[r] - ptr[r0];
    blocks->offsets.push_back(std::move(off));
  }
  for (int b = 0; b < nblocks; ++b) {
    const std::int64_t r0 = blocks->row_begin[b];
    const std::int64_t r1 = blocks->row_begin[b + 1];
    const std::array<asc::extent_t, 2> shape{r1 - r0, cols};
    const auto& off = blocks->offsets[b];
    auto view = asc::CsrView<const T>::Create(
        off.data(), idx + ptr[r0], val + ptr[r0], shape, off.back(),
        asc::MemorySpace::kHost);
    if (!view.ok()) return nullptr;
    blocks->views.push_back(*view);
  }
  return blocks.release();
}

template <typename T>
int RunBlocks(void* handle, T alpha, const T* x, T beta, T* y) {
  auto* blocks = static_cast<Blocks<T>*>(handle);
  const int n = static_cast<int>(blocks->views.size());
  std::vector<int> codes(static_cast<std::size_t>(n), 0);
  auto work = [&](int b) {
    const std::int64_t r0 = blocks->row_begin[b];
    const std::int64_t r1 = blocks->row_begin[b + 1];
    const HarnessVector<const T> in{x, blocks->cols, 1};
    HarnessVector<T> out{y + r0, r1 - r0, 1};
    codes[b] = Code(asc::Spmv(asc::ExecutionContext::Serial(), alpha,
                              blocks->views[b], in, beta, out));
  };
  if (n == 1) {
    work(0);
  } else {
    std::vector<std::thread> threads;
    for (int b = 0; b < n; ++b) threads.emplace_back(work, b);
    for (auto& t : threads) t.join();
  }
  for (int c : codes) {
    if (c != 0) return c;
  }
  return 0;
}

// Copies a reference-owned compressed array out to caller buffers
// (outer offsets [outer+1], inner indices [nnz], values [nnz]).
template <typename Array, typename T>
int CopyOut(Array& array, std::int64_t outer, std::int64_t* out_ptr,
            std::int64_t* out_idx, T* out_val) {
  auto view = array.view();
  if (!view.ok()) return Code(view.status());
  const std::int64_t nnz = view->nnz();
  std::copy(view->outer_offsets(), view->outer_offsets() + outer + 1, out_ptr);
  std::copy(view->inner_indices(), view->inner_indices() + nnz, out_idx);
  std::copy(view->values(), view->values() + nnz, out_val);
  return 0;
}

// to_csc = 1: CSR arrays in, CSC arrays out; 0: CSC in, CSR out.
template <typename T>
int ConvertCompressed(int to_csc, std::int64_t rows, std::int64_t cols,
                      const std::int64_t* ptr, const std::int64_t* idx,
                      const T* val, std::int64_t nnz, std::int64_t* out_ptr,
                      std::int64_t* out_idx, T* out_val) {
  const std::array<asc::extent_t, 2> shape{rows, cols};
  asc::HostMemoryResource resource;
  const auto context = asc::ExecutionContext::Serial();
  if (to_csc) {
    auto src = asc::CsrView<const T>::Create(ptr, idx, val, shape, nnz,
                                             asc::MemorySpace::kHost);
    if (!src.ok()) return Code(src.status());
    auto dst = asc::ConvertToCsc<const T>(context, *src, resource);
    if (!dst.ok()) return Code(dst.status());
    return CopyOut(*dst, cols, out_ptr, out_idx, out_val);
  }
  auto src = asc::CscView<const T>::Create(ptr, idx, val, shape, nnz,
                                           asc::MemorySpace::kHost);
  if (!src.ok()) return Code(src.status());
  auto dst = asc::ConvertToCsr<const T>(context, *src, resource);
  if (!dst.ok()) return Code(dst.status());
  return CopyOut(*dst, rows, out_ptr, out_idx, out_val);
}

// Canonical coordinates (interleaved [nnz][2]) to CSR (to_csc = 0) or CSC.
template <typename T>
int ConvertCoordinates(int to_csc, std::int64_t rows, std::int64_t cols,
                       const std::int64_t* coordinates, const T* val,
                       std::int64_t nnz, std::int64_t* out_ptr,
                       std::int64_t* out_idx, T* out_val) {
  const std::array<asc::extent_t, 2> shape{rows, cols};
  asc::HostMemoryResource resource;
  const auto context = asc::ExecutionContext::Serial();
  auto src = asc::CoordinateView<const T, 2>::Create(
      coordinates, val, std::span<const asc::extent_t, 2>(shape), nnz,
      asc::MemorySpace::kHost);
  if (!src.ok()) return Code(src.status());
  if (to_csc) {
    auto dst = asc::ConvertToCsc<const T>(context, *src, resource);
    if (!dst.ok()) return Code(dst.status());
    return CopyOut(*dst, cols, out_ptr, out_idx, out_val);
  }
  auto dst = asc::ConvertToCsr<const T>(context, *src, resource);
  if (!dst.ok()) return Code(dst.status());
  return CopyOut(*dst, rows, out_ptr, out_idx, out_val);
}

template <typename T, typename R>
T MakeScalar(R re, R im) {
  if constexpr (sizeof(T) == 2 * sizeof(R)) {
    return T(re, im);
  } else {
    (void)im;
    return T(re);
  }
}

// Level-1 on an indexed vector through the reference's SparseDot /
// SparseAxpy / SparseGather / SparseGatherZero / SparseScatter
// (blas.h:1340-1600).  op: 0 dot, 1 axpy, 2 gather, 3 gather-zero,
// 4 scatter; x is the dense vector (unit stride), result receives the dot.
template <typename T>
int Level1(int op, int conj, const std::int64_t* idx, T* val, std::int64_t nnz,
           std::int64_t n, T alpha, T* x, T* result) {
  const asc::ConstMemoryView idx_storage{idx, static_cast<std::size_t>(nnz) * 8,
                                         asc::MemorySpace::kHost};
  const asc::ConstMemoryView val_storage{val, static_cast<std::size_t>(nnz) * sizeof(T),
                                         asc::MemorySpace::kHost};
  const asc::ConstMemoryView x_const{x, static_cast<std::size_t>(n) * sizeof(T),
                                     asc::MemorySpace::kHost};
  const asc::MutableMemoryView x_mut{x, static_cast<std::size_t>(n) * sizeof(T),
                                     asc::MemorySpace::kHost};
  const auto context = asc::ExecutionContext::Serial();
  if (op == 0 || op == 1 || op == 4) {
    auto sparse = asc::SparseBlasIndexedVectorView<const T>::Create(idx, val, nnz, n, idx_storage,
                                                                    val_storage);
    if (!sparse.ok()) return Code(sparse.status());
    if (op == 0) {
      auto dense = asc::SparseBlasVectorView<const T>::Create(x, n, 1, x_const);
      if (!dense.ok()) return Code(dense.status());
      auto r = asc::SparseDot(context,
                              conj ? asc::SparseBlasConjugation::kConjugated
                                   : asc::SparseBlasConjugation::kUnconjugated,
                              *sparse, *dense);
      if (!r.ok()) return Code(r.status());
      *result = *r;
      return 0;
    }
    auto dense = asc::SparseBlasVectorView<T>::Create(x, n, 1, x_mut);
    if (!dense.ok()) return Code(dense.status());
    return op == 1 ? Code(asc::SparseAxpy(context, alpha, *sparse, *dense))
                   : Code(asc::SparseScatter(context, *sparse, *dense));
  }
  auto sparse = asc::SparseBlasIndexedVectorView<T>::Create(idx, val, nnz, n, idx_storage,
                                                            val_storage);
  if (!sparse.ok()) return Code(sparse.status());
  if (op == 2) {
    auto dense = asc::SparseBlasVectorView<const T>::Create(x, n, 1, x_const);
    if (!dense.ok()) return Code(dense.status());
    return Code(asc::SparseGather(context, *dense, *sparse));
  }
  auto dense = asc::SparseBlasVectorView<T>::Create(x, n, 1, x_mut);
  if (!dense.ok()) return Code(dense.status());
  return Code(asc::SparseGatherZero(context, *dense, *sparse));
}

// Sparse triangular solve through the reference's SparseBlasTriangularView
// (blas.h:1074-1160, which checks the triangle and, for a non-unit diagonal,
// that every diagonal entry is stored and nonzero) and
// SparseTriangularSolveMultiple (blas.h:1856-1910) on the n x k dense
// right-hand sides b (layout 0 column major, 1 row major), solved in place.
template <typename T>
int TriangularSolve(int op, int triangle, int diagonal, std::int64_t n,
                    const std::int64_t* ptr, const std::int64_t* idx, const T* val,
                    std::int64_t nnz, T alpha, T* b, int layout, std::int64_t ld,
                    std::int64_t k, std::size_t b_storage) {
  const std::array<asc::extent_t, 2> shape{n, n};
  auto m = asc::CsrView<const T>::Create(ptr, idx, val, shape, nnz, asc::MemorySpace::kHost);
  if (!m.ok()) return Code(m.status());
  auto tri = asc::SparseBlasTriangularView<T, asc::SparseCompressedFormat::kCsr>::Create(
      *m, static_cast<asc::SparseBlasTriangle>(triangle),
      static_cast<asc::SparseBlasDiagonal>(diagonal));
  if (!tri.ok()) return Code(tri.status());
  auto rhs = asc::SparseBlasMatrixView<T>::Create(
      b, n, k, static_cast<asc::SparseBlasLayout>(layout), ld,
      asc::MutableMemoryView(b, b_storage * sizeof(T), asc::MemorySpace::kHost));
  if (!rhs.ok()) return Code(rhs.status());
  return Code(asc::SparseTriangularSolveMultiple(asc::ExecutionContext::Serial(), Op(op), alpha,
                                                 *tri, *rhs));
}

}  // namespace

extern "C" {

int ref_compat_spmv_f64(std::int64_t rows, std::int64_t cols,
                        const std::int64_t* ptr, const std::int64_t* idx,
                        const double* val, std::int64_t nnz, double alpha,
                        const double* x, std::int64_t incx, double beta,
                        double* y, std::int64_t incy) {
  return CompatSpmv<double>(rows, cols, ptr, idx, val, nnz, alpha, x, incx,
                            beta, y, incy);
}

int ref_compat_spmv_f32(std::int64_t rows, std::int64_t cols,
                        const std::int64_t* ptr, const std::int64_t* idx,
                        const float* val, std::int64_t nnz, float alpha,
                        const float* x, std::int64_t incx, float beta, float* y,
                        std::int64_t incy) {
  return CompatSpmv<float>(rows, cols, ptr, idx, val, nnz, alpha, x, incx,
                           beta, y, incy);
}

// format: 1 = CSR, 2 = CSC.  op: 0 none, 1 transpose, 2 conjugate transpose.
#define ASC_REF_STANDARD(SUFFIX, T)                                            \
  int ref_standard_spmv_##SUFFIX(                                              \
      int format, int op, std::int64_t rows, std::int64_t cols,                \
      const std::int64_t* ptr, const std::int64_t* idx, const T* val,          \
      std::int64_t nnz, T alpha, const T* x, std::int64_t nx,                  \
      std::int64_t incx, std::size_t x_storage, T* y, std::int64_t ny,         \
      std::int64_t incy, std::size_t y_storage) {                              \
    if (format == 2) {                                                         \
      return StandardSpmvTyped<T, asc::SparseCompressedFormat::kCsc>(          \
          op, rows, cols, ptr, idx, val, nnz, alpha, x, nx, incx, x_storage,   \
          y, ny, incy, y_storage);                                             \
    }                                                                          \
    return StandardSpmvTyped<T, asc::SparseCompressedFormat::kCsr>(            \
        op, rows, cols, ptr, idx, val, nnz, alpha, x, nx, incx, x_storage, y,  \
        ny, incy, y_storage);                                                  \
  }                                                                            \
  int ref_standard_spmm_##SUFFIX(                                              \
      int format, int op, std::int64_t rows, std::int64_t cols,                \
      const std::int64_t* ptr, const std::int64_t* idx, const T* val,          \
      std::int64_t nnz, T alpha, const T* b, std::int64_t b_rows,              \
      std::int64_t b_cols, int b_layout, std::int64_t ldb,                     \
      std::size_t b_storage, T* c, std::int64_t c_rows, std::int64_t c_cols,   \
      int c_layout, std::int64_t ldc, std::size_t c_storage) {                 \
    if (format == 2) {                                                         \
      return StandardSpmmTyped<T, asc::SparseCompressedFormat::kCsc>(          \
          op, rows, cols, ptr, idx, val, nnz, alpha, b, b_rows, b_cols,        \
          b_layout, ldb, b_storage, c, c_rows, c_cols, c_layout, ldc,          \
          c_storage);                                                          \
    }                                                                          \
    return StandardSpmmTyped<T, asc::SparseCompressedFormat::kCsr>(            \
        op, rows, cols, ptr, idx, val, nnz, alpha, b, b_rows, b_cols,          \
        b_layout, ldb, b_storage, c, c_rows, c_cols, c_layout, ldc,            \
        c_storage);                                                            \
  }

ASC_REF_STANDARD(f64, double)
ASC_REF_STANDARD(f32, float)
#undef ASC_REF_STANDARD

// Complex element kinds: arrays are interleaved (re, im) pairs, the layout of
// std::complex<R>; alpha arrives as its two parts.
#define ASC_REF_COMPLEX(SUFFIX, R)                                             \
  int ref_standard_spmv_##SUFFIX(                                              \
      int format, int op, std::int64_t rows, std::int64_t cols,                \
      const std::int64_t* ptr, const std::int64_t* idx, const R* val,          \
      std::int64_t nnz, R alpha_re, R alpha_im, const R* x, std::int64_t nx,   \
      std::int64_t incx, std::size_t x_storage, R* y, std::int64_t ny,         \
      std::int64_t incy, std::size_t y_storage) {                              \
    using C = std::complex<R>;                                                 \
    const auto* v = reinterpret_cast<const C*>(val);                           \
    const auto* xc = reinterpret_cast<const C*>(x);                            \
    auto* yc = reinterpret_cast<C*>(y);                                        \
    const C alpha(alpha_re, alpha_im);                                         \
    if (format == 2) {                                                         \
      return StandardSpmvTyped<C, asc::SparseCompressedFormat::kCsc>(          \
          op, rows, cols, ptr, idx, v, nnz, alpha, xc, nx, incx, x_storage,    \
          yc, ny, incy, y_storage);                                            \
    }                                                                          \
    return StandardSpmvTyped<C, asc::SparseCompressedFormat::kCsr>(            \
        op, rows, cols, ptr, idx, v, nnz, alpha, xc, nx, incx, x_storage, yc,  \
        ny, incy, y_storage);                                                  \
  }                                                                            \
  int ref_standard_spmm_##SUFFIX(                                              \
      int format, int op, std::int64_t rows, std::int64_t cols,                \
      const std::int64_t* ptr, const std::int64_t* idx, const R* val,          \
      std::int64_t nnz, R alpha_re, R alpha_im, const R* b,                    \
      std::int64_t b_rows, std::int64_t b_cols, int b_layout,                  \
      std::int64_t ldb, std::size_t b_storage, R* c, std::int64_t c_rows,      \
      std::int64_t c_cols, int c_layout, std::int64_t ldc,                     \
      std::size_t c_storage) {                                                 \
    using C = std::complex<R>;                                                 \
    const auto* v = reinterpret_cast<const C*>(val);                           \
    const C alpha(alpha_re, alpha_im);                                         \
    const auto* bc = reinterpret_cast<const C*>(b);                            \
    auto* cc = reinterpret_cast<C*>(c);                                        \
    if (format == 2) {                                                         \
      return StandardSpmmTyped<C, asc::SparseCompressedFormat::kCsc>(          \
          op, rows, cols, ptr, idx, v, nnz, alpha, bc, b_rows, b_cols,         \
          b_layout, ldb, b_storage, cc, c_rows, c_cols, c_layout, ldc,         \
          c_storage);                                                          \
    }                                                                          \
    return StandardSpmmTyped<C, asc::SparseCompressedFormat::kCsr>(            \
        op, rows, cols, ptr, idx, v, nnz, alpha, bc, b_rows, b_cols, b_layout, \
        ldb, b_storage, cc, c_rows, c_cols, c_layout, ldc, c_storage);         \
  }

ASC_REF_COMPLEX(z, double)
ASC_REF_COMPLEX(c, float)
#undef ASC_REF_COMPLEX

void* ref_blocks_prepare_f64(std::int64_t rows, std::int64_t cols,
                             const std::int64_t* ptr, const std::int64_t* idx,
                             const double* val, int nblocks) {
  return PrepareBlocks<double>(rows, cols, ptr, idx, val, nblocks);
}
void* ref_blocks_prepare_f32(std::int64_t rows, std::int64_t cols,
                             const std::int64_t* ptr, const std::int64_t* idx,
                             const float* val, int nblocks) {
  return PrepareBlocks<float>(rows, cols, ptr, idx, val, nblocks);
}
int ref_blocks_run_f64(void* h, double alpha, const double* x, double beta,
                       double* y) {
  return RunBlocks<double>(h, alpha, x, beta, y);
}
int ref_blocks_run_f32(void* h, float alpha, const float* x, float beta,
                       float* y) {
  return RunBlocks<float>(h, alpha, x, beta, y);
}
void ref_blocks_free_f64(void* h) { delete static_cast<Blocks<double>*>(h); }
void ref_blocks_free_f32(void* h) { delete static_cast<Blocks<float>*>(h); }

int ref_convert_compressed_f64(int to_csc, std::int64_t rows,
                               std::int64_t cols, const std::int64_t* ptr,
                               const std::int64_t* idx, const double* val,
                               std::int64_t nnz, std::int64_t* out_ptr,
                               std::int64_t* out_idx, double* out_val) {
  return ConvertCompressed<double>(to_csc, rows, cols, ptr, idx, val, nnz,
                                   out_ptr, out_idx, out_val);
}
int ref_convert_coordinates_f64(int to_csc, std::int64_t rows,
                                std::int64_t cols,
                                const std::int64_t* coordinates,
                                const double* val, std::int64_t nnz,
                                std::int64_t* out_ptr, std::int64_t* out_idx,
                                double* out_val) {
  return ConvertCoordinates<double>(to_csc, rows, cols, coordinates, val, nnz,
                                    out_ptr, out_idx, out_val);
}

#define ASC_REF_LEVEL1(SUFFIX, T, R)                                            \
  int ref_level1_##SUFFIX(int op, int conj, const std::int64_t* idx, R* val,    \
                          std::int64_t nnz, std::int64_t n, R alpha_re,         \
                          R alpha_im, R* x, R* result) {                        \
    const T alpha = MakeScalar<T>(alpha_re, alpha_im);                          \
    return Level1<T>(op, conj, idx, reinterpret_cast<T*>(val), nnz, n, alpha,   \
                     reinterpret_cast<T*>(x), reinterpret_cast<T*>(result));    \
  }
ASC_REF_LEVEL1(f64, double, double)
ASC_REF_LEVEL1(f32, float, float)
ASC_REF_LEVEL1(z, std::complex<double>, double)
ASC_REF_LEVEL1(c, std::complex<float>, float)
#undef ASC_REF_LEVEL1

#define ASC_REF_TRSV(SUFFIX, T, R)                                              \
  int ref_trsv_##SUFFIX(int op, int triangle, int diagonal, std::int64_t n,     \
                        const std::int64_t* ptr, const std::int64_t* idx,       \
                        const R* val, std::int64_t nnz, R alpha_re, R alpha_im, \
                        R* b, int layout, std::int64_t ld, std::int64_t k,      \
                        std::size_t b_storage) {                                \
    return TriangularSolve<T>(op, triangle, diagonal, n, ptr, idx,              \
                              reinterpret_cast<const T*>(val), nnz,             \
                              MakeScalar<T>(alpha_re, alpha_im),                \
                              reinterpret_cast<T*>(b), layout, ld, k,           \
                              b_storage);                                       \
  }
ASC_REF_TRSV(f64, double, double)
ASC_REF_TRSV(f32, float, float)
ASC_REF_TRSV(z, std::complex<double>, double)
ASC_REF_TRSV(c, std::complex<float>, float)
#undef ASC_REF_TRSV

}  // extern "C"
