// Pointwise evaluation over one sparsity structure: asc_sb_evaluate.
//
// The reference's sparse expression evaluator on CUDA (EvaluateErased,
// src/sparse/cuda/operations.cc:1051-1120) copies, negates, adds, subtracts or
// multiplies the value arrays of operands that share the destination's
// structure (or scalars), one stored position at a time.  It is not a hot
// path; it is here so that every exported function of the reference's CUDA
// provider has a counterpart behind this library.  Validation follows the
// reference's rules and error codes, and runs before anything is enqueued.
#include <cuda_runtime.h>

#include <cstdint>
#include <limits>
#include <mutex>
#include <string>

#include "../../include/asc_sparse_b200.h"
#include "host/context_view.h"
#include "host/validate.h"

namespace {

using ascb::host::Fail;
using ascb::host::Span;
using ascb::host::Status;

struct Operand {
  const void* values;  // nullptr: scalar
  double scalar;
};

template <typename T>
__device__ __forceinline__ T read(const Operand& o, int64_t p) {
  return o.values != nullptr ? static_cast<const T*>(o.values)[p] : static_cast<T>(o.scalar);
}

template <typename T>
__global__ void __launch_bounds__(256) pointwise_kernel(int op, Operand left, Operand right,
                                                        T* __restrict__ out, int64_t n) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += step) {
    const T a = read<T>(left, p);
    T v = a;
    switch (op) {
      case ASC_SB_POINTWISE_NEGATE: v = -a; break;
      case ASC_SB_POINTWISE_ADD: v = a + read<T>(right, p); break;
      case ASC_SB_POINTWISE_SUBTRACT: v = a - read<T>(right, p); break;
      case ASC_SB_POINTWISE_MULTIPLY: v = a * read<T>(right, p); break;
      default: break;  // copy
    }
    out[p] = v;
  }
}

struct TensorBytes {
  std::size_t first = 0, second = 0, values = 0;
};

bool MulOverflows(std::uint64_t a, std::uint64_t b, std::uint64_t* out) {
  return __builtin_mul_overflow(a, b, out);
}

// ValidateSparseMetadata (operations.cc:134-251) for a descriptor of any rank.
Status TensorMetadata(const asc_sb_tensor& t, TensorBytes* out) {
  if (t.rank < 0 || (t.rank != 0 && t.extents == nullptr)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA operand extents are missing");
  }
  if (t.format != ASC_SB_COORDINATE && t.format != ASC_SB_CSR && t.format != ASC_SB_CSC) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA operand format is invalid");
  }
  if (t.element_kind < ASC_SB_FLOAT || t.element_kind > ASC_SB_COMPLEX_DOUBLE) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA scalar kind is invalid");
  }
  bool empty = false;
  std::uint64_t logical = 1;
  for (int64_t d = 0; d < t.rank; ++d) {
    if (t.extents[d] < 0) return Fail(ASC_SB_SHAPE, "A sparse CUDA extent cannot be negative");
    empty = empty || t.extents[d] == 0;
    if (!empty && (MulOverflows(logical, static_cast<std::uint64_t>(t.extents[d]), &logical) ||
                   logical > static_cast<std::uint64_t>(std::numeric_limits<int64_t>::max()))) {
      return Fail(ASC_SB_OVERFLOW, "Sparse CUDA shape overflows");
    }
  }
  if (empty) logical = 0;
  if (t.nonzeros < 0 || static_cast<std::uint64_t>(t.nonzeros) > logical) {
    return Fail(ASC_SB_SHAPE, "Sparse CUDA NNZ is incompatible with its shape");
  }
  if (!t.canonical_structure_trusted) {
    return Fail(ASC_SB_INVALID_ARGUMENT,
                "Sparse CUDA operations require trusted canonical structure");
  }
  const auto nnz = static_cast<std::uint64_t>(t.nonzeros);
  TensorBytes b;
  std::uint64_t v = 0;
  if (MulOverflows(nnz, ascb::host::ElementBytes(t.element_kind), &v)) {
    return Fail(ASC_SB_OVERFLOW, "Sparse CUDA storage size overflows");
  }
  b.values = v;
  if (t.format == ASC_SB_COORDINATE) {
    std::uint64_t count = 0, bytes = 0;
    if (MulOverflows(nnz, static_cast<std::uint64_t>(t.rank), &count) ||
        MulOverflows(count, 8, &bytes)) {
      return Fail(ASC_SB_OVERFLOW, "Sparse CUDA storage size overflows");
    }
    b.first = bytes;
  } else {
    if (t.rank != 2) return Fail(ASC_SB_SHAPE, "Compressed sparse CUDA operands require rank two");
    const int64_t outer = t.format == ASC_SB_CSR ? t.extents[0] : t.extents[1];
    std::uint64_t first = 0, second = 0;
    if (outer == std::numeric_limits<int64_t>::max() ||
        MulOverflows(static_cast<std::uint64_t>(outer) + 1, 8, &first) ||
        MulOverflows(nnz, 8, &second)) {
      return Fail(ASC_SB_OVERFLOW, "Sparse CUDA storage size overflows");
    }
    b.first = first;
    b.second = second;
  }
  const std::size_t value_align = t.element_kind == ASC_SB_FLOAT ||
                                          t.element_kind == ASC_SB_COMPLEX_FLOAT
                                      ? 4
                                      : 8;
  Status s = ascb::host::ValidateAddress(t.structure_first, b.first, 8,
                                         "Sparse CUDA structure storage is incomplete",
                                         "Sparse CUDA structure storage is misaligned");
  if (!s.ok()) return s;
  s = ascb::host::ValidateAddress(t.structure_second, b.second, 8,
                                  "Sparse CUDA index storage is incomplete",
                                  "Sparse CUDA index storage is misaligned");
  if (!s.ok()) return s;
  s = ascb::host::ValidateAddress(t.values, b.values, value_align,
                                  "Sparse CUDA value storage is incomplete",
                                  "Sparse CUDA value storage is misaligned");
  if (!s.ok()) return s;
  const Span first{t.structure_first, b.first}, second{t.structure_second, b.second},
      values{t.values, b.values};
  if (ascb::host::Overlap(first, second) || ascb::host::Overlap(first, values) ||
      ascb::host::Overlap(second, values)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA descriptor storage spans cannot overlap");
  }
  *out = b;
  return Status::Ok();
}

// ValidateSparseDevice (operations.cc:253-275).
Status TensorDevice(const asc_sb_tensor& t, int device, TensorBytes* out) {
  if (t.memory_space != ASC_SB_DEVICE) {
    return Fail(ASC_SB_MEMORY_ACCESS, "Sparse CUDA operations require device storage");
  }
  TensorBytes b;
  Status s = TensorMetadata(t, &b);
  if (!s.ok()) return s;
  for (const Span& span : {Span{t.structure_first, b.first}, Span{t.structure_second, b.second},
                           Span{t.values, b.values}}) {
    s = ascb::host::ValidateDevicePointer(span.begin, span.bytes, device,
                                          "CUDA could not inspect sparse operand storage");
    if (!s.ok()) return s;
  }
  if (out != nullptr) *out = b;
  return Status::Ok();
}

// SameStructure + ValidateEvaluationOperand (operations.cc:494-535).
Status OperandValid(const asc_sb_operand& o, const asc_sb_tensor& dst, int device) {
  if (o.kind == ASC_SB_OPERAND_SCALAR) {
    if (o.view.element_kind != dst.element_kind) {
      return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse scalar type does not match destination");
    }
    return Status::Ok();
  }
  if (o.kind != ASC_SB_OPERAND_VIEW) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse operand kind is invalid");
  }
  if (o.view.element_kind != dst.element_kind) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse value types do not match");
  }
  Status s = TensorDevice(o.view, device, nullptr);
  if (!s.ok()) return s;
  const asc_sb_tensor& v = o.view;
  if (v.format != dst.format || v.rank != dst.rank || v.nonzeros != dst.nonzeros ||
      v.structure_first != dst.structure_first || v.structure_second != dst.structure_second) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse evaluation requires identical structure");
  }
  for (int64_t d = 0; d < v.rank; ++d) {
    if (v.extents[d] != dst.extents[d]) {
      return Fail(ASC_SB_SHAPE, "CUDA sparse evaluation shapes do not match");
    }
  }
  return Status::Ok();
}

class Guard {
 public:
  explicit Guard(int device) {
    ok_ = cudaGetDevice(&previous_) == cudaSuccess &&
          (previous_ == device || cudaSetDevice(device) == cudaSuccess);
    if (!ok_) (void)cudaGetLastError();
  }
  ~Guard() {
    int now = -1;
    if (ok_ && cudaGetDevice(&now) == cudaSuccess && now != previous_) (void)cudaSetDevice(previous_);
  }
  bool ok() const { return ok_; }

 private:
  int previous_ = 0;
  bool ok_ = false;
};

int Done(const ascb::host::ContextView& v, const Status& s) {
  *v.last_error = s.ok() ? std::string() : s.message;
  return s.code;
}

Operand AsOperand(const asc_sb_operand& o) {
  return {o.kind == ASC_SB_OPERAND_VIEW ? o.view.values : nullptr, o.scalar};
}

}  // namespace

extern "C" ASC_SB_API int asc_sb_evaluate(asc_sb_context* context, int32_t operation,
                                          const asc_sb_operand* left,
                                          const asc_sb_operand* right,
                                          const asc_sb_tensor* destination) {
  using ascb::host::ContextView;
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  const bool binary = operation == ASC_SB_POINTWISE_ADD || operation == ASC_SB_POINTWISE_SUBTRACT ||
                      operation == ASC_SB_POINTWISE_MULTIPLY;
  if (operation < ASC_SB_POINTWISE_COPY || operation > ASC_SB_POINTWISE_MULTIPLY) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse pointwise operation is invalid"));
  }
  if (left == nullptr || destination == nullptr || (binary && right == nullptr)) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse evaluation operands cannot be null"));
  }
  TensorBytes db;
  Status s = TensorDevice(*destination, v.device, &db);
  if (!s.ok()) return Done(v, s);
  s = OperandValid(*left, *destination, v.device);
  if (!s.ok()) return Done(v, s);
  if (binary) {
    s = OperandValid(*right, *destination, v.device);
    if (!s.ok()) return Done(v, s);
  }
  for (const asc_sb_operand* o : {left, binary ? right : nullptr}) {
    if (o == nullptr || o->kind != ASC_SB_OPERAND_VIEW) continue;
    TensorBytes ob;
    s = TensorMetadata(o->view, &ob);
    if (!s.ok()) return Done(v, s);
    if (o->view.values != destination->values &&
        ascb::host::Overlap({o->view.values, ob.values}, {destination->values, db.values})) {
      return Done(v, Fail(ASC_SB_INVALID_ARGUMENT,
                          "CUDA sparse evaluation rejects partial value overlap"));
    }
  }
  if (destination->element_kind != ASC_SB_FLOAT && destination->element_kind != ASC_SB_DOUBLE) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT,
                        "CUDA sparse evaluation supports float and double values"));
  }
  if (destination->nonzeros == 0) return Done(v, Status::Ok());
  const int64_t n = destination->nonzeros;
  int64_t blocks = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(v.sm_count > 0 ? v.sm_count : 148) * 8;
  if (blocks > cap) blocks = cap;
  const Operand a = AsOperand(*left);
  const Operand b = binary ? AsOperand(*right) : Operand{nullptr, 0.0};
  void* out = const_cast<void*>(destination->values);
  if (destination->element_kind == ASC_SB_FLOAT) {
    pointwise_kernel<float><<<static_cast<unsigned>(blocks), 256, 0, v.stream>>>(
        operation, a, b, static_cast<float*>(out), n);
  } else {
    pointwise_kernel<double><<<static_cast<unsigned>(blocks), 256, 0, v.stream>>>(
        operation, a, b, static_cast<double*>(out), n);
  }
  v.launches->fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    (void)cudaStreamSynchronize(v.stream);
    (void)cudaGetLastError();
    return Done(v, {ASC_SB_PROVIDER,
                    std::string("CUDA could not launch the sparse pointwise kernel: ") +
                        cudaGetErrorString(e)});
  }
  return Done(v, Status::Ok());
}
