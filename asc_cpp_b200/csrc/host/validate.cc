// Host-side operand validation; rules and codes follow the reference provider
// (src/sparse/cuda/operations.cc), re-expressed over the C descriptors.
#include "validate.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <limits>

namespace ascb::host {
namespace {

// Checked a*b for non-negative 64-bit operands.
bool MulOverflows(std::uint64_t a, std::uint64_t b, std::uint64_t* out) {
  return __builtin_mul_overflow(a, b, out);
}

std::size_t ElementAlignment(int kind) {
  switch (kind) {
    case ASC_SB_FLOAT: return alignof(float);
    case ASC_SB_DOUBLE: return alignof(double);
    case ASC_SB_COMPLEX_FLOAT: return alignof(float);
    case ASC_SB_COMPLEX_DOUBLE: return alignof(double);
    default: return 1;
  }
}

bool KnownKind(int kind) { return kind >= ASC_SB_FLOAT && kind <= ASC_SB_COMPLEX_DOUBLE; }

}  // namespace

std::size_t ElementBytes(int kind) {
  switch (kind) {
    case ASC_SB_FLOAT: return 4;
    case ASC_SB_DOUBLE: return 8;
    case ASC_SB_COMPLEX_FLOAT: return 8;
    case ASC_SB_COMPLEX_DOUBLE: return 16;
    default: return 0;
  }
}

bool Overlap(Span a, Span b) {
  if (a.bytes == 0 || b.bytes == 0) return false;
  const auto ab = reinterpret_cast<std::uintptr_t>(a.begin);
  const auto bb = reinterpret_cast<std::uintptr_t>(b.begin);
  if (a.bytes > UINTPTR_MAX - ab || b.bytes > UINTPTR_MAX - bb) return true;
  return ab < bb + b.bytes && bb < ab + a.bytes;
}

Status ValidateAddress(const void* p, std::size_t bytes, std::size_t alignment,
                       const char* null_message, const char* align_message) {
  if (bytes == 0) return Status::Ok();
  if (p == nullptr) return Fail(ASC_SB_INVALID_ARGUMENT, null_message);
  const auto address = reinterpret_cast<std::uintptr_t>(p);
  if (address % alignment != 0) return Fail(ASC_SB_MEMORY_ACCESS, align_message);
  if (bytes > UINTPTR_MAX - address) {
    return Fail(ASC_SB_OVERFLOW, "A sparse CUDA operand address span overflows");
  }
  return Status::Ok();
}

Status ValidateDevicePointer(const void* p, std::size_t bytes, int device,
                             const char* message) {
  if (bytes == 0) return Status::Ok();
  cudaPointerAttributes attributes{};
  const cudaError_t error = cudaPointerGetAttributes(&attributes, p);
  if (error != cudaSuccess) {
    (void)cudaGetLastError();
    return Fail(ASC_SB_MEMORY_ACCESS, message);
  }
  if (attributes.type != cudaMemoryTypeDevice || attributes.device != device) {
    return Fail(ASC_SB_MEMORY_ACCESS,
                "A sparse CUDA operand is not on the context device");
  }
  return Status::Ok();
}

Status ValidateSparse(const asc_sb_sparse& m, int device, SparseBytes* out) {
  if (m.memory_space != ASC_SB_DEVICE) {
    return Fail(ASC_SB_MEMORY_ACCESS, "Sparse CUDA operations require device storage");
  }
  SparseBytes b;
  Status s = ValidateSparseMetadata(m, &b);
  if (!s.ok()) return s;
  for (const Span& span : {Span{m.structure_first, b.first}, Span{m.structure_second, b.second},
                           Span{m.values, b.values}}) {
    s = ValidateDevicePointer(span.begin, span.bytes, device,
                              "CUDA could not inspect sparse operand storage");
    if (!s.ok()) return s;
  }
  if (out) *out = b;
  return Status::Ok();
}

Status ValidateSparseMetadata(const asc_sb_sparse& m, SparseBytes* out) {
  if (m.format != ASC_SB_CSR && m.format != ASC_SB_CSC) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA SpMV/SpMM requires CSR or CSC format");
  }
  if (!KnownKind(m.element_kind)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA scalar kind is invalid");
  }
  if (m.rows < 0 || m.columns < 0) {
    return Fail(ASC_SB_SHAPE, "A sparse CUDA extent cannot be negative");
  }
  std::uint64_t logical = 0;
  if (m.rows != 0 && m.columns != 0 &&
      MulOverflows(static_cast<std::uint64_t>(m.rows),
                   static_cast<std::uint64_t>(m.columns), &logical)) {
    return Fail(ASC_SB_OVERFLOW, "Sparse CUDA shape overflows");
  }
  if (m.nonzeros < 0 || static_cast<std::uint64_t>(m.nonzeros) > logical) {
    return Fail(ASC_SB_SHAPE, "Sparse CUDA NNZ is incompatible with its shape");
  }
  if (!m.canonical_structure_trusted) {
    return Fail(ASC_SB_INVALID_ARGUMENT,
                "Sparse CUDA operations require trusted canonical structure");
  }
  const std::int64_t outer = m.format == ASC_SB_CSR ? m.rows : m.columns;
  SparseBytes b;
  std::uint64_t v = 0;
  if (MulOverflows(static_cast<std::uint64_t>(m.nonzeros), ElementBytes(m.element_kind), &v) ||
      MulOverflows(static_cast<std::uint64_t>(outer) + 1, 8, &b.first) ||
      MulOverflows(static_cast<std::uint64_t>(m.nonzeros), 8, &b.second)) {
    return Fail(ASC_SB_OVERFLOW, "Sparse CUDA storage size overflows");
  }
  b.values = v;
  Status s = ValidateAddress(m.structure_first, b.first, 8,
                             "Sparse CUDA structure storage is incomplete",
                             "Sparse CUDA structure storage is misaligned");
  if (!s.ok()) return s;
  s = ValidateAddress(m.structure_second, b.second, 8,
                      "Sparse CUDA index storage is incomplete",
                      "Sparse CUDA index storage is misaligned");
  if (!s.ok()) return s;
  s = ValidateAddress(m.values, b.values, ElementAlignment(m.element_kind),
                      "Sparse CUDA value storage is incomplete",
                      "Sparse CUDA value storage is misaligned");
  if (!s.ok()) return s;
  const Span first{m.structure_first, b.first};
  const Span second{m.structure_second, b.second};
  const Span values{m.values, b.values};
  if (Overlap(first, second) || Overlap(first, values) || Overlap(second, values)) {
    return Fail(ASC_SB_INVALID_ARGUMENT,
                "Sparse CUDA descriptor storage spans cannot overlap");
  }
  if (out) *out = b;
  return Status::Ok();
}

Status ValidateVector(const asc_sb_vector& v, int kind, bool writable,
                      int device, Span* span) {
  if (v.element_kind != kind || (v.writable != 0) != writable) {
    return Fail(ASC_SB_INVALID_ARGUMENT,
                "Sparse CUDA vector type or mutability is incorrect");
  }
  if (v.memory_space != ASC_SB_DEVICE) {
    return Fail(ASC_SB_MEMORY_ACCESS, "Sparse CUDA vectors require device storage");
  }
  if (v.extent < 0 || v.stride == 0) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA vector metadata is invalid");
  }
  Span touched{v.data, 0};
  if (v.extent > 0) {
    if (v.stride == std::numeric_limits<std::int64_t>::min()) {
      return Fail(ASC_SB_OVERFLOW, "Sparse CUDA vector stride magnitude overflows");
    }
    const std::uint64_t magnitude =
        static_cast<std::uint64_t>(v.stride < 0 ? -v.stride : v.stride);
    std::uint64_t last = 0, count = 0, bytes = 0;
    if (MulOverflows(static_cast<std::uint64_t>(v.extent - 1), magnitude, &last) ||
        __builtin_add_overflow(last, 1, &count) ||
        MulOverflows(count, ElementBytes(kind), &bytes)) {
      return Fail(ASC_SB_OVERFLOW, "Sparse CUDA vector span overflows");
    }
    touched.bytes = bytes;
    if (v.stride < 0) {
      // data is logical element 0, the highest address of the span
      const auto hi = reinterpret_cast<std::uintptr_t>(v.data);
      const std::uint64_t back = last * ElementBytes(kind);
      if (back > hi) return Fail(ASC_SB_OVERFLOW, "Sparse CUDA vector span overflows");
      touched.begin = reinterpret_cast<const void*>(hi - back);
    }
  }
  const void* check_ptr = v.reachable_data ? v.reachable_data : touched.begin;
  const std::size_t check_bytes = v.reachable_size ? v.reachable_size : touched.bytes;
  Status s = ValidateAddress(touched.bytes ? check_ptr : nullptr, touched.bytes ? check_bytes : 0,
                             ElementAlignment(kind),
                             "A nonempty sparse CUDA vector cannot be null",
                             "A sparse CUDA vector is misaligned");
  if (!s.ok()) return s;
  if (touched.bytes) {
    s = ValidateAddress(v.data, 1, ElementAlignment(kind),
                        "A nonempty sparse CUDA vector cannot be null",
                        "A sparse CUDA vector is misaligned");
    if (!s.ok()) return s;
  }
  s = ValidateDevicePointer(check_ptr, touched.bytes ? check_bytes : 0, device,
                            "CUDA could not inspect a sparse vector");
  if (!s.ok()) return s;
  if (span) *span = touched;
  return Status::Ok();
}

Status ValidateDense(const asc_sb_dense& d, int kind, bool writable,
                     int device, Span* span) {
  if (d.rows < 0 || d.columns < 0 || d.element_kind != kind ||
      (d.writable != 0) != writable || d.memory_space != ASC_SB_DEVICE ||
      (d.layout != ASC_SB_COLUMN_MAJOR && d.layout != ASC_SB_ROW_MAJOR)) {
    return Fail(ASC_SB_INVALID_ARGUMENT,
                "A CUDA Sparse BLAS dense-matrix descriptor is invalid");
  }
  const std::int64_t contiguous = d.layout == ASC_SB_COLUMN_MAJOR ? d.rows : d.columns;
  const bool vector_like = d.layout == ASC_SB_ROW_MAJOR && d.columns == 1;
  if ((!vector_like && d.leading_dimension < std::max<std::int64_t>(1, contiguous)) ||
      (vector_like && d.leading_dimension == 0)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "A CUDA Sparse BLAS leading dimension is too small");
  }
  Span touched{d.data, 0};
  if (d.rows != 0 && d.columns != 0) {
    if (d.leading_dimension == std::numeric_limits<std::int64_t>::min()) {
      return Fail(ASC_SB_OVERFLOW, "Dense matrix leading dimension overflows");
    }
    const std::int64_t major = d.layout == ASC_SB_COLUMN_MAJOR ? d.columns : d.rows;
    const std::uint64_t magnitude = static_cast<std::uint64_t>(
        d.leading_dimension < 0 ? -d.leading_dimension : d.leading_dimension);
    std::uint64_t lead = 0, total = 0, bytes = 0;
    if (MulOverflows(static_cast<std::uint64_t>(major - 1), magnitude, &lead) ||
        __builtin_add_overflow(lead, static_cast<std::uint64_t>(contiguous), &total) ||
        MulOverflows(total, ElementBytes(kind), &bytes)) {
      return Fail(ASC_SB_OVERFLOW, "Dense matrix span overflows");
    }
    touched.bytes = bytes;
    if (d.leading_dimension < 0) {
      const auto hi = reinterpret_cast<std::uintptr_t>(d.data);
      const std::uint64_t back = lead * ElementBytes(kind);
      if (back > hi) return Fail(ASC_SB_OVERFLOW, "Dense matrix span overflows");
      touched.begin = reinterpret_cast<const void*>(hi - back);
    }
  }
  const void* check_ptr = d.reachable_data ? d.reachable_data : touched.begin;
  const std::size_t check_bytes = d.reachable_size ? d.reachable_size : touched.bytes;
  Status s = ValidateAddress(touched.bytes ? check_ptr : nullptr, touched.bytes ? check_bytes : 0,
                             ElementAlignment(kind),
                             "A nonempty CUDA Sparse BLAS matrix cannot be null",
                             "A CUDA Sparse BLAS matrix is misaligned");
  if (!s.ok()) return s;
  s = ValidateDevicePointer(check_ptr, touched.bytes ? check_bytes : 0, device,
                            "CUDA could not inspect a Sparse BLAS dense matrix");
  if (!s.ok()) return s;
  if (span) *span = touched;
  return Status::Ok();
}

}  // namespace ascb::host
