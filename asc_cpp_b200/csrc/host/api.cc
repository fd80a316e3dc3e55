// C++20 host implementation of include/asc_sparse_b200.h.
//
// Mirrors the reference provider's control flow (src/sparse/cuda/
// operations.cc): validate the context, guard the device, validate every
// operand (including cudaPointerGetAttributes placement checks and overlap
// rules), and only then enqueue kernels on the context stream.  A failure after
// an enqueue synchronizes the stream before returning.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "../../../include/asc_sparse_b200.h"
#include "../kernels.h"
#include "context_view.h"
#include "validate.h"

using ascb::host::Fail;
using ascb::host::Span;
using ascb::host::SparseBytes;
using ascb::host::Status;

struct asc_sb_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  int determinism = ASC_SB_DETERMINISTIC;
  int variant = ASC_SB_VARIANT_AUTO;
  int lanes = 0;
  int sm_count = 148;
  std::mutex mutex;
  std::string last_error;
  std::atomic<std::int64_t> launches{0};
  int* status = nullptr;  // device word: kernels record bounded-wait timeouts
};

// Partitions of one CSR structure, as the kernels consume them.
struct Partitions {
  const std::int64_t* warp_tiles = nullptr;    // ascb_row_tiles, warp-tile weights
  std::int64_t n_warp = 0;
  const std::int64_t* merge_bounds = nullptr;  // ascb_merge_bounds pairs
  std::int64_t n_merge = 0;
};

struct asc_sb_plan {
  asc_sb_sparse matrix{};
  int flags = 0;
  Partitions part;    // of the stored arrays read as CSR
  // transposed structure (CSR of the transpose of the stored arrays)
  std::int64_t* t_ptr = nullptr;
  std::int64_t* t_idx = nullptr;
  void* t_val = nullptr;
  std::int64_t* t_perm = nullptr;
  Partitions t_part;
};

namespace {

constexpr std::size_t kWorkspaceAlignment = 16;  // alignof(std::max_align_t)

std::size_t RoundUp(std::size_t v, std::size_t a) { return (v + a - 1) / a * a; }

class DeviceGuard {
 public:
  explicit DeviceGuard(int device) {
    ok_ = cudaGetDevice(&previous_) == cudaSuccess &&
          (previous_ == device || cudaSetDevice(device) == cudaSuccess);
    if (!ok_) (void)cudaGetLastError();
  }
  ~DeviceGuard() {
    int now = -1;
    if (ok_ && cudaGetDevice(&now) == cudaSuccess && now != previous_) {
      (void)cudaSetDevice(previous_);
    }
  }
  bool ok() const { return ok_; }

 private:
  int previous_ = 0;
  bool ok_ = false;
};

int Finish(asc_sb_context* ctx, const Status& s) {
  if (ctx != nullptr) ctx->last_error = s.ok() ? std::string() : s.message;
  return s.code;
}

// Launch result -> status; after a failed enqueue the stream is drained so the
// caller can release operands safely (operations.cc:1027-1045).
Status Launched(asc_sb_context* ctx, int err, const char* message) {
  ctx->launches.fetch_add(1, std::memory_order_relaxed);
  if (err == 0) return Status::Ok();
  (void)cudaStreamSynchronize(ctx->stream);
  (void)cudaGetLastError();
  return {ASC_SB_PROVIDER,
          std::string(message) + ": " + cudaGetErrorString(static_cast<cudaError_t>(err))};
}

int Dtype(int kind) { return kind == ASC_SB_DOUBLE ? ASCB_F64 : ASCB_F32; }

bool RealKind(int kind) { return kind == ASC_SB_FLOAT || kind == ASC_SB_DOUBLE; }

ascb_csr AsCsr(const asc_sb_sparse& m, bool swap_shape) {
  ascb_csr a{};
  a.rows = swap_shape ? m.columns : m.rows;
  a.cols = swap_shape ? m.rows : m.columns;
  a.nnz = m.nonzeros;
  a.ptr = static_cast<const std::int64_t*>(m.structure_first);
  a.idx = static_cast<const std::int64_t*>(m.structure_second);
  a.val = m.values;
  return a;
}

ascb_vec AsVec(const asc_sb_vector& v) {
  return ascb_vec{const_cast<void*>(v.data), v.extent, v.stride};
}

Status ValidateContext(asc_sb_context* ctx) {
  if (ctx == nullptr) {
    return Fail(ASC_SB_INVALID_STATE, "A null or moved-from Sparse CUDA context cannot launch work");
  }
  if (ctx->stream == nullptr && !ctx->owns_stream) {
    // the legacy default stream is allowed only when explicitly chosen
  }
  return Status::Ok();
}

// Number of warp row tiles of a CSR structure.
std::int64_t WarpTiles(std::int64_t rows, std::int64_t nnz) {
  return ascb_row_tile_count(rows, nnz, ascb_warp_tile_items(), ascb_warp_tile_row_weight());
}
std::size_t WarpTileBytes(std::int64_t rows, std::int64_t nnz) {
  return RoundUp(static_cast<std::size_t>(WarpTiles(rows, nnz) + 1) * 8, 256);
}
std::size_t MergeBoundBytes(std::int64_t rows, std::int64_t nnz) {
  return RoundUp(static_cast<std::size_t>(ascb_merge_tiles(rows, nnz) + 1) * 16, 256);
}

// ---- workspace layout of asc_sb_csr_spmv ----------------------------------
// The size is a function of the matrix shape only, so it is stable for a given
// (A, x, y) (the reference's rule, operations.cc:884-909): room for the
// partition of whichever kernel the context selects.
std::size_t CompatWorkspaceBytes(const asc_sb_sparse& m) {
  if (m.rows == 0 || m.columns == 0) return 0;
  return std::max(WarpTileBytes(m.rows, m.nonzeros), MergeBoundBytes(m.rows, m.nonzeros));
}

// Choice of SpMV kernel for a real CSR product.
struct Choice {
  int variant = ASC_SB_VARIANT_ROW_ORDERED;
  int lanes = 0;
};

int AutoLanes(const asc_sb_sparse& m, bool transposed_rows) {
  const std::int64_t rows = transposed_rows ? m.columns : m.rows;
  const double mean = rows > 0 ? static_cast<double>(m.nonzeros) / static_cast<double>(rows) : 0.0;
  int lanes = 1;
  while (lanes < 32 && lanes * 2 <= mean) lanes *= 2;
  return lanes;
}

Choice Choose(const asc_sb_context* ctx, const asc_sb_sparse& m) {
  Choice c;
  if (ctx->determinism == ASC_SB_DETERMINISTIC) return c;  // bit-exact order
  if (ctx->variant != ASC_SB_VARIANT_AUTO) {
    c.variant = ctx->variant;
    c.lanes = ctx->lanes > 0 ? ctx->lanes : AutoLanes(m, false);
    return c;
  }
  c.variant = ASC_SB_VARIANT_WARP_TILES;
  return c;
}

// Runs one real CSR SpMV with the chosen kernel.  Partitions come from the
// plan when there is one, else are built into `scratch` (caller workspace),
// else the kernel that searches its own tile bounds is used.
Status RunCsr(asc_sb_context* ctx, const Choice& choice, int form,
              const ascb_csr& a, int dtype, double alpha, double beta,
              const ascb_vec& x, const ascb_vec& y, std::int64_t* scratch,
              const Partitions* planned) {
  if (choice.variant == ASC_SB_VARIANT_VECTOR) {
    const int lanes = choice.lanes > 0 ? choice.lanes : 4;
    return Launched(ctx,
                    ascb_spmv_vector(ctx->stream, dtype, form, lanes, &a, alpha, beta, &x, &y,
                                     ctx->sm_count),
                    "CUDA could not launch the vector CSR SpMV kernel");
  }
  const int exact = choice.variant == ASC_SB_VARIANT_ROW_ORDERED ? 1 : 0;
  if (choice.variant == ASC_SB_VARIANT_MERGE_PATH) {
    const std::int64_t tiles = ascb_merge_tiles(a.rows, a.nnz);
    const std::int64_t* bounds = planned != nullptr ? planned->merge_bounds : nullptr;
    if (bounds == nullptr && scratch != nullptr) {
      Status s = Launched(ctx, ascb_merge_bounds(ctx->stream, &a, scratch, tiles),
                          "CUDA could not launch the merge partition kernel");
      if (!s.ok()) return s;
      bounds = scratch;
    }
    if (bounds != nullptr) {
      return Launched(ctx,
                      ascb_spmv_merge(ctx->stream, dtype, form, exact, &a, alpha, beta, &x, &y,
                                      bounds, tiles, ctx->sm_count, ctx->status),
                      "CUDA could not launch the merge SpMV kernel");
    }
    // no partition buffer at all (zero-workspace calls): warp tiles with
    // in-kernel bound search
  }
  const std::int64_t tiles = WarpTiles(a.rows, a.nnz);
  const std::int64_t* tiles_ptr = planned != nullptr ? planned->warp_tiles : nullptr;
  if (tiles_ptr == nullptr && scratch != nullptr) {
    Status s = Launched(ctx,
                        ascb_row_tiles(ctx->stream, &a, ascb_warp_tile_items(),
                                       ascb_warp_tile_row_weight(), scratch, tiles),
                        "CUDA could not launch the row-tile partition kernel");
    if (!s.ok()) return s;
    tiles_ptr = scratch;
  }
  // ROW_ORDERED (bit-exact) and WARP_TILES (contracted) run the register-
  // segmented kernel, which needs 16-byte aligned index and value arrays;
  // otherwise the scalar-load warp kernel with the same numerics.
  const bool seg_aligned =
      ((reinterpret_cast<std::uintptr_t>(a.idx) | reinterpret_cast<std::uintptr_t>(a.val)) &
       static_cast<std::uintptr_t>(ascb_spmv_seg_alignment() - 1)) == 0;
  if (seg_aligned) {
    return Launched(ctx,
                    ascb_spmv_seg(ctx->stream, dtype, form, exact, &a, alpha, beta, &x, &y,
                                  tiles_ptr, tiles, ctx->sm_count),
                    "CUDA could not launch the segmented SpMV kernel");
  }
  return Launched(ctx,
                  ascb_spmv_warp(ctx->stream, dtype, form, exact, &a, alpha, beta, &x, &y,
                                 tiles_ptr, tiles, ctx->sm_count),
                  "CUDA could not launch the warp-tiled SpMV kernel");
}

// Builds both partitions of `a` into `buffer` (plan memory).
Status BuildPartitions(asc_sb_context* ctx, const ascb_csr& a, unsigned char* buffer,
                       Partitions* out) {
  out->n_warp = WarpTiles(a.rows, a.nnz);
  out->n_merge = ascb_merge_tiles(a.rows, a.nnz);
  auto* warp = reinterpret_cast<std::int64_t*>(buffer);
  auto* merge = reinterpret_cast<std::int64_t*>(buffer + WarpTileBytes(a.rows, a.nnz));
  out->warp_tiles = warp;
  out->merge_bounds = merge;
  if (a.rows == 0) return Status::Ok();
  Status s = Launched(ctx,
                      ascb_row_tiles(ctx->stream, &a, ascb_warp_tile_items(),
                                     ascb_warp_tile_row_weight(), warp, out->n_warp),
                      "CUDA could not launch the row-tile partition kernel");
  if (!s.ok()) return s;
  return Launched(ctx, ascb_merge_bounds(ctx->stream, &a, merge, out->n_merge),
                  "CUDA could not launch the merge partition kernel");
}
std::size_t PartitionBytes(std::int64_t rows, std::int64_t nnz) {
  return WarpTileBytes(rows, nnz) + MergeBoundBytes(rows, nnz);
}

struct CompatOperands {
  SparseBytes matrix_bytes;
  Span x_span, y_span;
};

Status ValidateCompat(asc_sb_context* ctx, const asc_sb_sparse* m,
                      const asc_sb_vector* x, const asc_sb_vector* y,
                      CompatOperands* out) {
  if (m == nullptr || x == nullptr || y == nullptr) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV descriptors cannot be null");
  }
  if (m->format != ASC_SB_CSR) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV requires CSR format");
  }
  Status s = ascb::host::ValidateSparse(*m, ctx->device, &out->matrix_bytes);
  if (!s.ok()) return s;
  if (!RealKind(m->element_kind)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV supports float and double");
  }
  s = ascb::host::ValidateVector(*x, m->element_kind, false, ctx->device, &out->x_span);
  if (!s.ok()) return s;
  s = ascb::host::ValidateVector(*y, m->element_kind, true, ctx->device, &out->y_span);
  if (!s.ok()) return s;
  if (x->extent != m->columns || y->extent != m->rows) {
    return Fail(ASC_SB_SHAPE, "CUDA CSR SpMV vector lengths do not match the matrix");
  }
  const auto& b = out->matrix_bytes;
  if (ascb::host::Overlap(out->x_span, out->y_span) ||
      ascb::host::Overlap({m->structure_first, b.first}, out->y_span) ||
      ascb::host::Overlap({m->structure_second, b.second}, out->y_span) ||
      ascb::host::Overlap({m->values, b.values}, out->y_span)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV rejects output operand overlap");
  }
  return Status::Ok();
}

}  // namespace

extern "C" {

int asc_sb_context_create(int32_t device, void* stream, asc_sb_context** out) {
  if (out == nullptr) return ASC_SB_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    return ASC_SB_UNAVAILABLE;
  }
  if (device < 0 || device >= count) return ASC_SB_INVALID_ARGUMENT;
  DeviceGuard guard(device);
  if (!guard.ok()) return ASC_SB_UNAVAILABLE;
  auto* ctx = new (std::nothrow) asc_sb_context();
  if (ctx == nullptr) return ASC_SB_ALLOCATION;
  ctx->device = device;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) {
    ctx->sm_count = sms;
  }
  if (stream == nullptr) {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      (void)cudaGetLastError();
      delete ctx;
      return ASC_SB_PROVIDER;
    }
    ctx->owns_stream = true;
  } else {
    ctx->stream = static_cast<cudaStream_t>(stream);
  }
  // One device word per context for kernels' bounded-wait timeouts (set-up
  // allocation; no operation allocates).
  if (cudaMalloc(reinterpret_cast<void**>(&ctx->status), sizeof(int)) != cudaSuccess ||
      cudaMemset(ctx->status, 0, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    if (ctx->owns_stream) (void)cudaStreamDestroy(ctx->stream);
    if (ctx->status != nullptr) (void)cudaFree(ctx->status);
    delete ctx;
    return ASC_SB_ALLOCATION;
  }
  *out = ctx;
  return ASC_SB_OK;
}

int asc_sb_context_destroy(asc_sb_context* ctx) {
  if (ctx == nullptr) return ASC_SB_OK;
  DeviceGuard guard(ctx->device);
  (void)cudaStreamSynchronize(ctx->stream);
  if (ctx->owns_stream) (void)cudaStreamDestroy(ctx->stream);
  if (ctx->status != nullptr) (void)cudaFree(ctx->status);
  delete ctx;
  return ASC_SB_OK;
}

int asc_sb_context_device_status(asc_sb_context* ctx, int32_t* value, int32_t clear) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  if (value == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "value cannot be null"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  int host = 0;
  cudaError_t e = cudaMemcpyAsync(&host, ctx->status, sizeof(int), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && clear) e = cudaMemsetAsync(ctx->status, 0, sizeof(int), ctx->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return Finish(ctx, {ASC_SB_PROVIDER, std::string("status read failed: ") + cudaGetErrorString(e)});
  }
  *value = host;
  return Finish(ctx, Status::Ok());
}

int asc_sb_context_set_determinism(asc_sb_context* ctx, int32_t determinism) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  if (determinism != ASC_SB_DETERMINISTIC && determinism != ASC_SB_BACKEND_DEFAULT) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Determinism is not a recognized enumerator"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->determinism = determinism;
  return ASC_SB_OK;
}

int asc_sb_context_set_variant(asc_sb_context* ctx, int32_t variant, int32_t lanes) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  const bool lanes_ok = lanes == 0 || (lanes > 0 && lanes <= 32 && (lanes & (lanes - 1)) == 0);
  if (variant < ASC_SB_VARIANT_AUTO || variant > ASC_SB_VARIANT_ROW_SPLIT || !lanes_ok) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Unknown SpMV variant or lane count"));
  }
  if (variant == ASC_SB_VARIANT_ROW_SPLIT) {
    return Finish(ctx, Fail(ASC_SB_UNSUPPORTED, "This SpMV variant is not available yet"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->variant = variant;
  ctx->lanes = lanes;
  return ASC_SB_OK;
}

void* asc_sb_context_stream(const asc_sb_context* ctx) {
  return ctx == nullptr ? nullptr : static_cast<void*>(ctx->stream);
}

int asc_sb_context_synchronize(asc_sb_context* ctx) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  DeviceGuard guard(ctx->device);
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return Finish(ctx, {ASC_SB_PROVIDER, std::string("stream synchronize failed: ") + cudaGetErrorString(e)});
  }
  return ASC_SB_OK;
}

const char* asc_sb_context_last_error(const asc_sb_context* ctx) {
  return ctx == nullptr ? "null context" : ctx->last_error.c_str();
}

int64_t asc_sb_context_launch_count(const asc_sb_context* ctx) {
  return ctx == nullptr ? 0 : ctx->launches.load(std::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
int asc_sb_csr_spmv_workspace_size(asc_sb_context* ctx, const asc_sb_sparse* m,
                                   const asc_sb_vector* x, const asc_sb_vector* y,
                                   size_t* bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (bytes == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "bytes cannot be null"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  CompatOperands ops;
  s = ValidateCompat(ctx, m, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  // Strided vectors (and empty shapes) take the zero-workspace path, as in
  // the reference (operations.cc:902-905).
  *bytes = (x->stride != 1 || y->stride != 1) ? 0 : CompatWorkspaceBytes(*m);
  return Finish(ctx, Status::Ok());
}

int asc_sb_csr_spmv(asc_sb_context* ctx, double alpha, const asc_sb_sparse* m,
                    const asc_sb_vector* x, double beta, const asc_sb_vector* y,
                    void* workspace, size_t workspace_bytes, int32_t workspace_space) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  CompatOperands ops;
  s = ValidateCompat(ctx, m, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (m->rows == 0) return Finish(ctx, Status::Ok());
  const bool strided = m->columns == 0 || x->stride != 1 || y->stride != 1;
  std::int64_t* tile_buffer = nullptr;
  if (strided) {
    if (workspace_bytes != 0) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                              "The strided CSR SpMV path requires zero workspace"));
    }
  } else {
    const std::size_t required = CompatWorkspaceBytes(*m);
    if (workspace_space != ASC_SB_DEVICE || workspace_bytes < required ||
        (required != 0 && workspace == nullptr)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                              "CUDA CSR SpMV workspace is missing or too small"));
    }
    s = ascb::host::ValidateAddress(workspace, workspace_bytes, kWorkspaceAlignment,
                                    "CUDA CSR SpMV workspace cannot be null",
                                    "CUDA CSR SpMV workspace is misaligned");
    if (!s.ok()) return Finish(ctx, s);
    s = ascb::host::ValidateDevicePointer(workspace, workspace_bytes, ctx->device,
                                          "CUDA could not inspect CSR SpMV workspace");
    if (!s.ok()) return Finish(ctx, s);
    const Span w{workspace, workspace_bytes};
    const auto& b = ops.matrix_bytes;
    if (ascb::host::Overlap(w, {m->structure_first, b.first}) ||
        ascb::host::Overlap(w, {m->structure_second, b.second}) ||
        ascb::host::Overlap(w, {m->values, b.values}) || ascb::host::Overlap(w, ops.x_span) ||
        ascb::host::Overlap(w, ops.y_span)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                              "CUDA CSR SpMV workspace overlaps an operand"));
    }
    tile_buffer = static_cast<std::int64_t*>(workspace);
  }
  const ascb_csr a = AsCsr(*m, false);
  const ascb_vec xv = AsVec(*x), yv = AsVec(*y);
  const Choice choice = Choose(ctx, *m);
  s = RunCsr(ctx, choice, ASCB_COMPAT, a, Dtype(m->element_kind), alpha, beta, xv, yv,
             tile_buffer, nullptr);
  return Finish(ctx, s);
}

// ---------------------------------------------------------------------------
namespace {

struct StandardOperands {
  SparseBytes matrix_bytes;
  Span in_span, out_span;
};

Status ValidateStandardSpmv(asc_sb_context* ctx, int op, double alpha_imag,
                            const asc_sb_sparse* m, const asc_sb_vector* x,
                            const asc_sb_vector* y, StandardOperands* out) {
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid");
  }
  if (m == nullptr || x == nullptr || y == nullptr) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA standardized SpMV descriptors cannot be null");
  }
  Status s = ascb::host::ValidateSparse(*m, ctx->device, &out->matrix_bytes);
  if (!s.ok()) return s;
  if (!RealKind(m->element_kind) || alpha_imag != 0.0) {
    return Fail(ASC_SB_UNSUPPORTED, "CUDA standardized SpMV supports real float and double");
  }
  s = ascb::host::ValidateVector(*x, m->element_kind, false, ctx->device, &out->in_span);
  if (!s.ok()) return s;
  s = ascb::host::ValidateVector(*y, m->element_kind, true, ctx->device, &out->out_span);
  if (!s.ok()) return s;
  const std::int64_t in_extent = op == ASC_SB_OP_NONE ? m->columns : m->rows;
  const std::int64_t out_extent = op == ASC_SB_OP_NONE ? m->rows : m->columns;
  if (x->extent != in_extent || y->extent != out_extent) {
    return Fail(ASC_SB_SHAPE, "CUDA standardized SpMV vector extents do not match");
  }
  const auto& b = out->matrix_bytes;
  if (ascb::host::Overlap(out->in_span, out->out_span) ||
      ascb::host::Overlap({m->structure_first, b.first}, out->out_span) ||
      ascb::host::Overlap({m->structure_second, b.second}, out->out_span) ||
      ascb::host::Overlap({m->values, b.values}, out->out_span)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA standardized SpMV output overlaps an input");
  }
  return Status::Ok();
}

// Runs y += alpha * op(A) x.  The stored arrays are read as a CSR matrix `a`
// (for CSC: the CSR of A^T); `transposed` says whether the product needs the
// transpose of those arrays.
Status RunStandardSpmv(asc_sb_context* ctx, const asc_sb_plan* plan,
                       const asc_sb_sparse& m, int op, double alpha,
                       const asc_sb_vector& x, const asc_sb_vector& y) {
  const bool csc = m.format == ASC_SB_CSC;
  const bool transposed = (op != ASC_SB_OP_NONE) != csc;
  const ascb_csr a = AsCsr(m, csc);
  const int dtype = Dtype(m.element_kind);
  const ascb_vec xv = AsVec(x), yv = AsVec(y);
  if (!transposed) {
    const Choice choice = Choose(ctx, m);
    return RunCsr(ctx, choice, ASCB_STANDARD, a, dtype, alpha, 0.0, xv, yv, nullptr,
                  plan != nullptr ? &plan->part : nullptr);
  }
  if (plan != nullptr && plan->t_ptr != nullptr) {
    ascb_csr t{};
    t.rows = a.cols;
    t.cols = a.rows;
    t.nnz = a.nnz;
    t.ptr = plan->t_ptr;
    t.idx = plan->t_idx;
    t.val = plan->t_val;
    const Choice choice = Choose(ctx, m);
    return RunCsr(ctx, choice, ASCB_STANDARD, t, dtype, alpha, 0.0, xv, yv, nullptr,
                  &plan->t_part);
  }
  if (ctx->determinism == ASC_SB_DETERMINISTIC) {
    return Fail(ASC_SB_INVALID_STATE,
                "A deterministic transposed product needs a plan created with "
                "ASC_SB_PLAN_TRANSPOSE");
  }
  return Launched(ctx, ascb_spmv_scatter(ctx->stream, dtype, &a, alpha, &xv, &yv, ctx->sm_count),
                  "CUDA could not launch the scatter SpMV kernel");
}

}  // namespace

int asc_sb_standard_spmv(asc_sb_context* ctx, int32_t op, double alpha_real, double alpha_imag,
                         const asc_sb_sparse* m, const asc_sb_vector* x, const asc_sb_vector* y) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  StandardOperands ops;
  s = ValidateStandardSpmv(ctx, op, alpha_imag, m, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (alpha_real == 0.0 || y->extent == 0) return Finish(ctx, Status::Ok());
  return Finish(ctx, RunStandardSpmv(ctx, nullptr, *m, op, alpha_real, *x, *y));
}

// ---------------------------------------------------------------------------
int asc_sb_standard_spmm(asc_sb_context* ctx, int32_t op, double alpha_real, double alpha_imag,
                         const asc_sb_sparse* m, const asc_sb_dense* b, const asc_sb_dense* c) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid"));
  }
  if (m == nullptr || b == nullptr || c == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "CUDA SpMM descriptors cannot be null"));
  }
  SparseBytes mb;
  s = ascb::host::ValidateSparse(*m, ctx->device, &mb);
  if (!s.ok()) return Finish(ctx, s);
  if (!RealKind(m->element_kind) || alpha_imag != 0.0) {
    return Finish(ctx, Fail(ASC_SB_UNSUPPORTED, "CUDA standardized SpMM supports real float and double"));
  }
  Span bs, cs;
  s = ascb::host::ValidateDense(*b, m->element_kind, false, ctx->device, &bs);
  if (!s.ok()) return Finish(ctx, s);
  s = ascb::host::ValidateDense(*c, m->element_kind, true, ctx->device, &cs);
  if (!s.ok()) return Finish(ctx, s);
  const std::int64_t inner = op == ASC_SB_OP_NONE ? m->columns : m->rows;
  const std::int64_t rows = op == ASC_SB_OP_NONE ? m->rows : m->columns;
  if (b->rows != inner || c->rows != rows || b->columns != c->columns) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "CUDA standardized SpMM matrix extents do not match"));
  }
  if (ascb::host::Overlap(bs, cs) || ascb::host::Overlap({m->structure_first, mb.first}, cs) ||
      ascb::host::Overlap({m->structure_second, mb.second}, cs) ||
      ascb::host::Overlap({m->values, mb.values}, cs)) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "CUDA standardized SpMM output overlaps an input"));
  }
  if (alpha_real == 0.0 || c->rows == 0 || c->columns == 0) return Finish(ctx, Status::Ok());
  const bool csc = m->format == ASC_SB_CSC;
  const bool transposed = (op != ASC_SB_OP_NONE) != csc;
  if (transposed && ctx->determinism == ASC_SB_DETERMINISTIC) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE,
                            "A deterministic transposed SpMM needs the transposed structure "
                            "(a CSR copy of A^T)"));
  }
  const ascb_csr a = AsCsr(*m, csc);
  s = Launched(ctx,
               ascb_spmm(ctx->stream, Dtype(m->element_kind), transposed ? 1 : 0, &a, c->columns,
                         b->data, b->layout, b->leading_dimension, const_cast<void*>(c->data),
                         c->layout, c->leading_dimension, alpha_real, ctx->sm_count),
               "CUDA could not launch the SpMM kernel");
  return Finish(ctx, s);
}

// ---------------------------------------------------------------------------
int asc_sb_plan_workspace_size(asc_sb_context* ctx, const asc_sb_sparse* m, int32_t flags,
                               size_t* bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (m == nullptr || bytes == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "plan arguments cannot be null"));
  }
  if (flags & ASC_SB_PLAN_TRANSPOSE) {
    return Finish(ctx, Fail(ASC_SB_UNSUPPORTED, "transposed plans are not built yet"));
  }
  const std::int64_t outer = m->format == ASC_SB_CSC ? m->columns : m->rows;
  *bytes = PartitionBytes(outer, m->nonzeros);
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_create(asc_sb_context* ctx, const asc_sb_sparse* m, int32_t flags,
                       void* workspace, size_t workspace_bytes, asc_sb_plan** out) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (m == nullptr || out == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "plan arguments cannot be null"));
  }
  *out = nullptr;
  size_t need = 0;
  int rc = asc_sb_plan_workspace_size(ctx, m, flags, &need);
  if (rc != ASC_SB_OK) return rc;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  SparseBytes mb;
  s = ascb::host::ValidateSparse(*m, ctx->device, &mb);
  if (!s.ok()) return Finish(ctx, s);
  if (workspace_bytes < need || (need != 0 && workspace == nullptr)) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "plan workspace is missing or too small"));
  }
  s = ascb::host::ValidateDevicePointer(workspace, workspace_bytes, ctx->device,
                                        "CUDA could not inspect plan workspace");
  if (!s.ok()) return Finish(ctx, s);
  auto* plan = new (std::nothrow) asc_sb_plan();
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_ALLOCATION, "plan allocation failed"));
  plan->matrix = *m;
  plan->flags = flags;
  const bool csc = m->format == ASC_SB_CSC;
  const ascb_csr a = AsCsr(*m, csc);
  s = BuildPartitions(ctx, a, static_cast<unsigned char*>(workspace), &plan->part);
  if (!s.ok()) {
    delete plan;
    return Finish(ctx, s);
  }
  *out = plan;
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_refresh_values(asc_sb_context* ctx, asc_sb_plan* plan) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_destroy(asc_sb_plan* plan) {
  delete plan;
  return ASC_SB_OK;
}

int asc_sb_plan_csr_spmv(asc_sb_context* ctx, const asc_sb_plan* plan, double alpha,
                         const asc_sb_vector* x, double beta, const asc_sb_vector* y) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  CompatOperands ops;
  s = ValidateCompat(ctx, &plan->matrix, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (plan->matrix.rows == 0) return Finish(ctx, Status::Ok());
  const ascb_csr a = AsCsr(plan->matrix, false);
  const Choice choice = Choose(ctx, plan->matrix);
  s = RunCsr(ctx, choice, ASCB_COMPAT, a, Dtype(plan->matrix.element_kind), alpha, beta,
             AsVec(*x), AsVec(*y), nullptr, &plan->part);
  return Finish(ctx, s);
}

int asc_sb_plan_standard_spmv(asc_sb_context* ctx, const asc_sb_plan* plan, int32_t op,
                              double alpha_real, double alpha_imag, const asc_sb_vector* x,
                              const asc_sb_vector* y) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  StandardOperands ops;
  s = ValidateStandardSpmv(ctx, op, alpha_imag, &plan->matrix, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (alpha_real == 0.0 || y->extent == 0) return Finish(ctx, Status::Ok());
  return Finish(ctx, RunStandardSpmv(ctx, plan, plan->matrix, op, alpha_real, *x, *y));
}

}  // extern "C"

namespace ascb::host {

bool ViewContext(asc_sb_context* ctx, ContextView* view) {
  if (ctx == nullptr || view == nullptr) return false;
  view->device = ctx->device;
  view->stream = ctx->stream;
  view->determinism = ctx->determinism;
  view->sm_count = ctx->sm_count;
  view->mutex = &ctx->mutex;
  view->last_error = &ctx->last_error;
  view->launches = &ctx->launches;
  return true;
}

}  // namespace ascb::host
