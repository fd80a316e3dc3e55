// Reference-side binding: the exported surface of ASCCpp's experimental
// sparse_cuda provider (include/asc/sparse/providers/cuda.h:212-253,499-606),
// implemented over this library's C ABI (include/asc_sparse_b200.h).
//
// A maintainer replaces src/sparse/cuda/{context.cc,operations.cc,kernels.cu}
// of the reference with this file and links libasc_sparse_b200.so; the
// reference's public headers do not change, so every caller of
// asc::CudaCsrSpmv / CudaSpmv / CudaSpmm / CudaCloneCsr / CudaEvaluate /
// CudaSparseDot / ... keeps working.  It is compiled against the reference's
// headers and its core internals (src/core/execution_internal.h for the
// execution context's native stream), exactly where the replaced files sat.
//
// Every function: checks the context the way the reference does
// (ValidateContext, operations.cc:51-75), converts the descriptors field for
// field, calls the C entry point (which validates everything before it
// enqueues, and drains the stream itself if an enqueue fails), and records
// the completion event on the execution context's stream
// (RecordCudaEvent, the reference's own completion path).
#include <cuda_runtime_api.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <utility>

#include "asc/core/providers/cuda.h"
#include "asc/sparse/providers/cuda.h"
#include "asc_sparse_b200.h"
#include "core/execution_internal.h"

namespace {
constexpr const char* kProvider = "asc_sparse_b200";  // Status::provider of library failures
}  // namespace

namespace asc::internal_sparse_cuda {

// Provider state: the library context bound to the execution context's
// stream.  Opaque to callers (cuda.h:102), so its layout is this binding's.
class ContextState {
 public:
  ContextState(std::int32_t device, asc_sb_context* b200) noexcept
      : device_(device), b200_(b200) {}
  ContextState(const ContextState&) = delete;
  ContextState& operator=(const ContextState&) = delete;
  ~ContextState() { static_cast<void>(asc_sb_context_destroy(b200_)); }

  [[nodiscard]] std::int32_t device() const noexcept { return device_; }
  [[nodiscard]] asc_sb_context* b200() const noexcept { return b200_; }

 private:
  std::int32_t device_;
  asc_sb_context* b200_;
};

namespace {

// ValidateContext (operations.cc:51-75): the library context, with the
// execution context's determinism applied for this call.
Result<asc_sb_context*> Bound(SparseCudaContext& context) {
  ContextState* state = Access::State(context);
  if (state == nullptr) {
    return Status(ErrorCode::kInvalidState, "A moved-from SparseCudaContext cannot launch work");
  }
  const ExecutionContext& execution = context.execution_context();
  if (execution.backend() != Backend::kCuda || execution.device().ordinal != state->device()) {
    return Status(ErrorCode::kInvalidState,
                  "Sparse CUDA provider state does not match its context");
  }
  const auto& execution_state = internal_core_execution::Access::State(execution);
  if (execution_state == nullptr) {
    return Status(ErrorCode::kInvalidState,
                  "The sparse CUDA execution context has no provider state");
  }
  if (execution_state->NativeExecutionHandle(Backend::kCuda) == nullptr) {
    return Status(ErrorCode::kUnavailable, "The sparse CUDA execution context has no stream");
  }
  static_cast<void>(asc_sb_context_set_determinism(
      state->b200(), static_cast<std::int32_t>(execution.determinism())));
  return state->b200();
}

Status FromC(int rc, asc_sb_context* c) {
  if (rc == ASC_SB_OK) return Status::Ok();
  return Status(static_cast<ErrorCode>(rc), asc_sb_context_last_error(c), kProvider, rc);
}

Result<CompletionEvent> Completed(int rc, asc_sb_context* c, SparseCudaContext& context) {
  if (rc != ASC_SB_OK) return FromC(rc, c);
  return RecordCudaEvent(context.execution_context());
}

std::int64_t Extent(const SparseDescriptor& d, std::size_t i, extent_t fallback) {
  return d.rank == 2 && d.extents != nullptr ? d.extents[i] : fallback;
}

asc_sb_sparse ToC(const SparseDescriptor& d) {
  asc_sb_sparse m{};
  m.structure_first = d.structure_first;
  m.structure_second = d.structure_second;
  m.values = d.values;
  m.memory_space = static_cast<std::int32_t>(d.memory_space);
  m.element_kind = static_cast<std::int32_t>(d.element_kind);
  m.format = static_cast<std::int32_t>(d.format);
  m.canonical_structure_trusted = d.canonical_structure_trusted ? 1 : 0;
  m.rows = Extent(d, 0, d.rows);
  m.columns = Extent(d, 1, d.columns);
  m.nonzeros = d.nonzeros;
  return m;
}

asc_sb_tensor ToTensor(const SparseDescriptor& d) {
  asc_sb_tensor t{};
  t.structure_first = d.structure_first;
  t.structure_second = d.structure_second;
  t.values = d.values;
  t.memory_space = static_cast<std::int32_t>(d.memory_space);
  t.element_kind = static_cast<std::int32_t>(d.element_kind);
  t.format = static_cast<std::int32_t>(d.format);
  t.canonical_structure_trusted = d.canonical_structure_trusted ? 1 : 0;
  t.rank = static_cast<std::int64_t>(d.rank);
  t.extents = d.extents;
  t.nonzeros = d.nonzeros;
  return t;
}

asc_sb_vector ToC(const VectorDescriptor& v) {
  asc_sb_vector c{};
  c.data = v.data;
  c.reachable_data = v.reachable_data;
  c.reachable_size = v.reachable_size;
  c.memory_space = static_cast<std::int32_t>(v.memory_space);
  c.element_kind = static_cast<std::int32_t>(v.element_kind);
  c.extent = v.extent;
  c.stride = v.stride;
  c.writable = v.writable ? 1 : 0;
  return c;
}

asc_sb_dense ToC(const MatrixDescriptor& m) {
  asc_sb_dense d{};
  d.data = m.data;
  d.reachable_data = m.reachable_data;
  d.reachable_size = m.reachable_size;
  d.memory_space = static_cast<std::int32_t>(m.memory_space);
  d.element_kind = static_cast<std::int32_t>(m.element_kind);
  d.rows = m.rows;
  d.columns = m.columns;
  d.leading_dimension = m.leading_dimension;
  d.layout = static_cast<std::int32_t>(m.layout);
  d.writable = m.writable ? 1 : 0;
  return d;
}

asc_sb_indexed_vector ToC(const IndexedVectorDescriptor& v) {
  asc_sb_indexed_vector c{};
  c.indices = v.indices;
  c.values = v.values;
  c.memory_space = static_cast<std::int32_t>(v.memory_space);
  c.element_kind = static_cast<std::int32_t>(v.element_kind);
  c.nonzeros = v.nonzeros;
  c.dense_extent = v.dense_extent;
  c.writable = v.writable ? 1 : 0;
  c.canonical_structure_trusted = v.canonical_structure_trusted ? 1 : 0;
  return c;
}

asc_sb_operand ToC(const OperandDescriptor& o) {
  asc_sb_operand c{};
  c.kind = o.kind == OperandKind::kView ? ASC_SB_OPERAND_VIEW : ASC_SB_OPERAND_SCALAR;
  c.view = ToTensor(o.view);
  c.scalar = o.scalar;
  return c;
}

std::size_t ElementAlignment(ElementKind kind) {
  return kind == ElementKind::kFloat || kind == ElementKind::kComplexFloat ? alignof(float)
                                                                           : alignof(double);
}

}  // namespace

Result<CloneBuffers> CloneCsrErased(SparseCudaContext& context, SparseDescriptor source,
                                    MemoryResource& resource) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  if (source.format != FormatKind::kCsr || source.memory_space != MemorySpace::kHost) {
    return Status(ErrorCode::kMemoryAccess, "CudaCloneCsr requires canonical host CSR storage");
  }
  const asc_sb_sparse host = ToC(source);
  std::size_t first = 0, second = 0, values = 0;
  int rc = asc_sb_sparse_storage_bytes(*c, &host, &first, &second, &values);
  if (rc != ASC_SB_OK) return FromC(rc, *c);
  if (resource.space() != MemorySpace::kDevice) {
    return Status(ErrorCode::kMemoryAccess, "CudaCloneCsr requires a device memory resource");
  }
  // the destination comes from the caller's resource, as in the reference
  auto offsets = Buffer::Allocate(resource, first, alignof(nnz_t));
  if (!offsets.ok()) return offsets.status();
  auto indices = Buffer::Allocate(resource, second, alignof(index_t));
  if (!indices.ok()) return indices.status();
  auto vals = Buffer::Allocate(resource, values, ElementAlignment(source.element_kind));
  if (!vals.ok()) return vals.status();
  asc_sb_sparse device = host;
  device.structure_first = offsets->data();
  device.structure_second = indices->data();
  device.values = vals->data();
  device.memory_space = ASC_SB_DEVICE;
  rc = asc_sb_clone_csr(*c, &host, &device);
  if (rc != ASC_SB_OK) return FromC(rc, *c);
  CompletionEvent completion = internal_core_execution::Access::MakeCompletedEvent();
  if (first + second + values != 0) {
    auto recorded = RecordCudaEvent(context.execution_context());
    if (!recorded.ok()) {
      static_cast<void>(asc_sb_context_synchronize(*c));
      return recorded.status();
    }
    completion = std::move(*recorded);
  }
  return CloneBuffers{.outer_offsets = std::move(*offsets),
                      .inner_indices = std::move(*indices),
                      .values = std::move(*vals),
                      .completion = std::move(completion)};
}

Result<IndexedCloneBuffers> CloneIndexedErased(SparseCudaContext& context,
                                               IndexedVectorDescriptor source,
                                               MemoryResource& resource) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  if (source.memory_space != MemorySpace::kHost) {
    return Status(ErrorCode::kMemoryAccess,
                  "CudaCloneIndexedVector requires a canonical host indexed vector");
  }
  const asc_sb_indexed_vector host = ToC(source);
  std::size_t index_bytes = 0, value_bytes = 0;
  int rc = asc_sb_indexed_storage_bytes(*c, &host, &index_bytes, &value_bytes);
  if (rc != ASC_SB_OK) return FromC(rc, *c);
  if (resource.space() != MemorySpace::kDevice) {
    return Status(ErrorCode::kMemoryAccess, "CudaCloneIndexedVector requires device memory");
  }
  auto indices = Buffer::Allocate(resource, index_bytes, alignof(index_t));
  if (!indices.ok()) return indices.status();
  auto values = Buffer::Allocate(resource, value_bytes, ElementAlignment(source.element_kind));
  if (!values.ok()) return values.status();
  asc_sb_indexed_vector device = host;
  device.indices = indices->data();
  device.values = values->data();
  device.memory_space = ASC_SB_DEVICE;
  device.writable = 1;
  rc = asc_sb_clone_indexed(*c, &host, &device);
  if (rc != ASC_SB_OK) return FromC(rc, *c);
  CompletionEvent completion = internal_core_execution::Access::MakeCompletedEvent();
  if (index_bytes + value_bytes != 0) {
    auto recorded = RecordCudaEvent(context.execution_context());
    if (!recorded.ok()) {
      static_cast<void>(asc_sb_context_synchronize(*c));
      return recorded.status();
    }
    completion = std::move(*recorded);
  }
  return IndexedCloneBuffers{.indices = std::move(*indices),
                             .values = std::move(*values),
                             .completion = std::move(completion)};
}

Result<std::size_t> CsrSpmvWorkspaceSizeErased(SparseCudaContext& context,
                                               SparseDescriptor matrix, VectorDescriptor input,
                                               VectorDescriptor output) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_sparse a = ToC(matrix);
  const asc_sb_vector x = ToC(input), y = ToC(output);
  std::size_t bytes = 0;
  const int rc = asc_sb_csr_spmv_workspace_size(*c, &a, &x, &y, &bytes);
  if (rc != ASC_SB_OK) return FromC(rc, *c);
  return bytes;
}

Result<CompletionEvent> CsrSpmvErased(SparseCudaContext& context, double alpha,
                                      SparseDescriptor matrix, VectorDescriptor input,
                                      double beta, VectorDescriptor output,
                                      MutableMemoryView workspace) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_sparse a = ToC(matrix);
  const asc_sb_vector x = ToC(input), y = ToC(output);
  const int rc = asc_sb_csr_spmv(*c, alpha, &a, &x, beta, &y, workspace.data(), workspace.size(),
                                 static_cast<std::int32_t>(workspace.space()));
  return Completed(rc, *c, context);
}

Result<CompletionEvent> EvaluateErased(SparseCudaContext& context, PointwiseOperation operation,
                                       OperandDescriptor left, OperandDescriptor right,
                                       SparseDescriptor destination) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_operand l = ToC(left), r = ToC(right);
  const asc_sb_tensor d = ToTensor(destination);
  const int rc = asc_sb_evaluate(*c, static_cast<std::int32_t>(operation), &l, &r, &d);
  if (rc == ASC_SB_OK && destination.nonzeros == 0) {
    return internal_core_execution::Access::MakeCompletedEvent();
  }
  return Completed(rc, *c, context);
}

Result<CompletionEvent> StandardLevel1Erased(SparseCudaContext& context,
                                             StandardOperation operation,
                                             SparseBlasConjugation conjugation, ScalarValue alpha,
                                             IndexedVectorDescriptor sparse,
                                             VectorDescriptor dense, VectorDescriptor result) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_indexed_vector s = ToC(sparse);
  const asc_sb_vector d = ToC(dense), r = ToC(result);
  const int rc = asc_sb_standard_level1(*c, static_cast<std::int32_t>(operation),
                                        static_cast<std::int32_t>(conjugation), alpha.real,
                                        alpha.imaginary, &s, &d, &r);
  return Completed(rc, *c, context);
}

Result<CompletionEvent> StandardSpmvErased(SparseCudaContext& context,
                                           SparseBlasTranspose transpose, ScalarValue alpha,
                                           SparseDescriptor matrix, VectorDescriptor input,
                                           VectorDescriptor output) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_sparse a = ToC(matrix);
  const asc_sb_vector x = ToC(input), y = ToC(output);
  const int rc = asc_sb_standard_spmv(*c, static_cast<std::int32_t>(transpose), alpha.real,
                                      alpha.imaginary, &a, &x, &y);
  return Completed(rc, *c, context);
}

Result<CompletionEvent> StandardSpmmErased(SparseCudaContext& context,
                                           SparseBlasTranspose transpose, ScalarValue alpha,
                                           SparseDescriptor matrix, MatrixDescriptor input,
                                           MatrixDescriptor output) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_sparse a = ToC(matrix);
  const asc_sb_dense b = ToC(input), out = ToC(output);
  const int rc = asc_sb_standard_spmm(*c, static_cast<std::int32_t>(transpose), alpha.real,
                                      alpha.imaginary, &a, &b, &out);
  return Completed(rc, *c, context);
}

Result<CompletionEvent> StandardTriangularSolveErased(SparseCudaContext& context,
                                                      SparseBlasTranspose transpose,
                                                      ScalarValue alpha, SparseDescriptor matrix,
                                                      SparseBlasTriangle triangle,
                                                      SparseBlasDiagonal diagonal,
                                                      MatrixDescriptor right_hand_sides) {
  auto c = Bound(context);
  if (!c.ok()) return c.status();
  const asc_sb_sparse a = ToC(matrix);
  const asc_sb_dense rhs = ToC(right_hand_sides);
  const int rc = asc_sb_standard_triangular_solve(
      *c, static_cast<std::int32_t>(transpose), alpha.real, alpha.imaginary, &a,
      static_cast<std::int32_t>(triangle), static_cast<std::int32_t>(diagonal), &rhs);
  return Completed(rc, *c, context);
}

}  // namespace asc::internal_sparse_cuda

namespace asc {

SparseCudaContext::SparseCudaContext(
    ExecutionContext execution_context,
    std::unique_ptr<internal_sparse_cuda::ContextState> state) noexcept
    : execution_context_(std::move(execution_context)), state_(std::move(state)) {}

SparseCudaContext::SparseCudaContext(SparseCudaContext&& other) noexcept = default;

SparseCudaContext& SparseCudaContext::operator=(SparseCudaContext&& other) noexcept {
  if (this != &other) {
    state_.reset();  // the old library context goes before the new one moves in
    execution_context_ = std::move(other.execution_context_);
    state_ = std::move(other.state_);
  }
  return *this;
}

SparseCudaContext::~SparseCudaContext() = default;

Result<SparseCudaContext> SparseCudaContext::Create(ExecutionContext execution_context) {
  if (execution_context.backend() != Backend::kCuda) {
    return Status(ErrorCode::kInvalidArgument,
                  "SparseCudaContext requires a CUDA execution context");
  }
  const auto& execution_state = internal_core_execution::Access::State(execution_context);
  if (execution_state == nullptr) {
    return Status(ErrorCode::kUnavailable, "The CUDA execution context has no provider state");
  }
  void* native_stream = execution_state->NativeExecutionHandle(Backend::kCuda);
  if (native_stream == nullptr) {
    return Status(ErrorCode::kUnavailable, "The CUDA execution context has no execution stream");
  }
  const std::int32_t device = execution_context.device().ordinal;
  asc_sb_context* b200 = nullptr;
  const int rc = asc_sb_context_create(device, native_stream, &b200);
  if (rc != ASC_SB_OK) {
    return Status(static_cast<ErrorCode>(rc), "The B200 sparse context could not be created",
                  kProvider, rc);
  }
  static_cast<void>(asc_sb_context_set_determinism(
      b200, static_cast<std::int32_t>(execution_context.determinism())));
  auto state = std::make_unique<internal_sparse_cuda::ContextState>(device, b200);
  return SparseCudaContext(std::move(execution_context), std::move(state));
}

}  // namespace asc
