// Batched compat SpMV: asc_sb_batch_* (no reference counterpart).
//
// A batch binds `count` independent CSR products y_i = alpha A_i x_i + beta y_i
// of one element kind.  Creation validates every operand with the same rules
// as asc_sb_csr_spmv, uploads a table of the operands and computes the row
// tiles of every matrix with one kernel; a product is then ONE launch of the
// persistent work-queue kernel (warps take tiles of any matrix from a global
// counter), optionally replayed from a CUDA graph.  The schedule -- tiles per
// queue grab and CTAs per SM -- is a parameter that asc_sb_batch_autotune
// chooses by timing.  asc_sb_batch_spmv_per_matrix runs the same products as
// one plain-kernel launch per matrix, the baseline the batch is measured
// against.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../../include/asc_sparse_b200.h"
#include "../kernels.h"
#include "context_view.h"
#include "validate.h"

using ascb::host::ContextView;
using ascb::host::Fail;
using ascb::host::Span;
using ascb::host::SparseBytes;
using ascb::host::Status;

struct asc_sb_batch {
  int device = 0;
  int element_kind = ASC_SB_DOUBLE;
  std::int64_t count = 0;
  bool unit = true;        // every vector has stride 1
  bool aligned = true;     // every index/value array is 16-byte aligned
  std::vector<ascb_batch_item> items;  // host copy (per-matrix path)
  ascb_batch_item* items_dev = nullptr;
  std::int64_t* bounds = nullptr;
  unsigned long long* queue = nullptr;
  std::int64_t total_tiles = 0;
  std::int64_t total_bounds = 0;
  int chunk = 4;
  int ctas_per_sm = 0;
  // captured graph and the launch it holds
  cudaGraphExec_t exec = nullptr;
  double g_alpha = 0.0, g_beta = 0.0;
  int g_chunk = 0, g_ctas = 0, g_exact = -1;
};

namespace {

constexpr std::size_t kAlign = 256;
std::size_t RoundUp(std::size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

int Done(const ContextView& v, const Status& s) {
  *v.last_error = s.ok() ? std::string() : s.message;
  return s.code;
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

std::int64_t Tiles(std::int64_t rows, std::int64_t nnz) {
  return ascb_row_tile_count(rows, nnz, ascb_warp_tile_items(), ascb_warp_tile_row_weight());
}

struct Layout {
  std::size_t items = 0, bounds = 0, queue = 0, total = 0;
  std::int64_t total_tiles = 0, total_bounds = 0;
};

Status LayoutFor(std::int64_t count, const asc_sb_sparse* m, Layout* out) {
  Layout l;
  for (std::int64_t i = 0; i < count; ++i) {
    if (m[i].rows < 0 || m[i].nonzeros < 0) return Fail(ASC_SB_SHAPE, "negative batch extents");
    const std::int64_t t = m[i].rows > 0 ? Tiles(m[i].rows, m[i].nonzeros) : 0;
    l.total_tiles += t;
    l.total_bounds += t + 1;
  }
  std::size_t at = 0;
  l.items = at;
  at += RoundUp(static_cast<std::size_t>(count) * sizeof(ascb_batch_item));
  l.bounds = at;
  at += RoundUp(static_cast<std::size_t>(l.total_bounds) * 8);
  l.queue = at;
  at += RoundUp(8);
  l.total = at;
  *out = l;
  return Status::Ok();
}

Status Enqueued(const ContextView& v, int err, const char* what) {
  v.launches->fetch_add(1, std::memory_order_relaxed);
  if (err == 0) return Status::Ok();
  (void)cudaStreamSynchronize(v.stream);
  (void)cudaGetLastError();
  return {ASC_SB_PROVIDER,
          std::string(what) + ": " + cudaGetErrorString(static_cast<cudaError_t>(err))};
}

int Dtype(int kind) { return kind == ASC_SB_DOUBLE ? ASCB_F64 : ASCB_F32; }

// Queue reset + persistent kernel on `stream` (also what a graph captures).
int EnqueuePersistent(cudaStream_t stream, const asc_sb_batch& b, int exact, double alpha,
                      double beta, int sm_count) {
  cudaError_t e = cudaMemsetAsync(b.queue, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return static_cast<int>(e);
  return ascb_spmv_seg_batch(stream, Dtype(b.element_kind), exact, b.unit ? 1 : 0, b.items_dev,
                             b.count, b.bounds, b.total_tiles, b.queue, b.chunk, b.ctas_per_sm,
                             alpha, beta, sm_count);
}

void DropGraph(asc_sb_batch* b) {
  if (b->exec != nullptr) (void)cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->g_exact = -1;
}

// One plain-kernel launch per matrix (the segmented kernel, or the scalar
// warp kernel for misaligned arrays) with the tile bounds computed at create.
Status PerMatrix(const ContextView& v, const asc_sb_batch& b, int exact, double alpha,
                 double beta) {
  for (const ascb_batch_item& it : b.items) {
    if (it.rows == 0) continue;
    ascb_csr a{};
    a.rows = it.rows;
    a.nnz = it.nnz;
    a.ptr = it.ptr;
    a.idx = it.idx;
    a.val = it.val;
    const ascb_vec x{const_cast<void*>(it.x), 0, it.incx};
    const ascb_vec y{it.y, it.rows, it.incy};
    const std::int64_t tiles = Tiles(it.rows, it.nnz);
    const std::int64_t* tb = b.bounds + it.bound_base;
    const bool aligned =
        ((reinterpret_cast<std::uintptr_t>(it.idx) | reinterpret_cast<std::uintptr_t>(it.val)) &
         static_cast<std::uintptr_t>(ascb_spmv_seg_alignment() - 1)) == 0;
    const int rc = aligned ? ascb_spmv_seg(v.stream, Dtype(b.element_kind), ASCB_COMPAT, exact, &a,
                                           alpha, beta, &x, &y, tb, tiles, v.sm_count)
                           : ascb_spmv_warp(v.stream, Dtype(b.element_kind), ASCB_COMPAT, exact,
                                            &a, alpha, beta, &x, &y, tb, tiles, v.sm_count);
    Status s = Enqueued(v, rc, "CUDA could not launch a per-matrix SpMV");
    if (!s.ok()) return s;
  }
  return Status::Ok();
}

Status RunBatch(const ContextView& v, asc_sb_batch* b, double alpha, double beta) {
  const int exact = v.determinism == ASC_SB_DETERMINISTIC ? 1 : 0;
  if (!b->aligned) return PerMatrix(v, *b, exact, alpha, beta);
  if (b->total_tiles == 0) return Status::Ok();
  if (b->exec != nullptr && b->g_alpha == alpha && b->g_beta == beta && b->g_exact == exact &&
      b->g_chunk == b->chunk && b->g_ctas == b->ctas_per_sm) {
    return Enqueued(v, static_cast<int>(cudaGraphLaunch(b->exec, v.stream)),
                    "CUDA could not launch the batch graph");
  }
  return Enqueued(v, EnqueuePersistent(v.stream, *b, exact, alpha, beta, v.sm_count),
                  "CUDA could not launch the batched SpMV");
}

// Products of a batch run concurrently, so no output may overlap another
// output, or any input or matrix array of the batch.
bool OutputsOverlap(std::vector<Span> writes, const std::vector<Span>& reads) {
  std::erase_if(writes, [](const Span& s) { return s.bytes == 0; });
  std::sort(writes.begin(), writes.end(), [](const Span& a, const Span& b) {
    return reinterpret_cast<std::uintptr_t>(a.begin) < reinterpret_cast<std::uintptr_t>(b.begin);
  });
  for (std::size_t i = 1; i < writes.size(); ++i) {
    if (ascb::host::Overlap(writes[i - 1], writes[i])) return true;
  }
  for (const Span& r : reads) {
    if (r.bytes == 0) continue;
    // the write spans are disjoint and sorted: if any of them overlaps r,
    // the last one that starts below r's end does
    const auto end = reinterpret_cast<std::uintptr_t>(r.begin) + r.bytes;
    auto it = std::lower_bound(writes.begin(), writes.end(), end,
                               [](const Span& w, std::uintptr_t e) {
                                 return reinterpret_cast<std::uintptr_t>(w.begin) < e;
                               });
    if (it != writes.begin() && ascb::host::Overlap(*(it - 1), r)) return true;
  }
  return false;
}

}  // namespace

extern "C" {

int asc_sb_batch_workspace_size(asc_sb_context* context, int64_t count,
                                const asc_sb_sparse* matrices, size_t* bytes) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (bytes == nullptr || count < 0 || (count > 0 && matrices == nullptr)) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch arguments are invalid"));
  }
  Layout l;
  Status s = LayoutFor(count, matrices, &l);
  if (s.ok()) *bytes = l.total;
  return Done(v, s);
}

int asc_sb_batch_create(asc_sb_context* context, int64_t count, const asc_sb_sparse* matrices,
                        const asc_sb_vector* inputs, const asc_sb_vector* outputs,
                        void* workspace, size_t workspace_bytes, asc_sb_batch** out) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (out == nullptr || count < 0 ||
      (count > 0 && (matrices == nullptr || inputs == nullptr || outputs == nullptr))) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch arguments are invalid"));
  }
  *out = nullptr;
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  Layout l;
  Status s = LayoutFor(count, matrices, &l);
  if (!s.ok()) return Done(v, s);
  auto b = std::make_unique<asc_sb_batch>();
  b->device = v.device;
  b->count = count;
  b->element_kind = count > 0 ? matrices[0].element_kind : ASC_SB_DOUBLE;
  b->items.resize(static_cast<std::size_t>(count));
  std::int64_t tile_base = 0;
  std::vector<Span> writes, reads;
  writes.reserve(static_cast<std::size_t>(count));
  reads.reserve(static_cast<std::size_t>(count) * 4);
  for (std::int64_t i = 0; i < count; ++i) {
    const asc_sb_sparse& m = matrices[i];
    if (m.format != ASC_SB_CSR) {
      return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batched SpMV requires CSR matrices"));
    }
    if (m.element_kind != b->element_kind ||
        (m.element_kind != ASC_SB_FLOAT && m.element_kind != ASC_SB_DOUBLE)) {
      return Done(v, Fail(ASC_SB_INVALID_ARGUMENT,
                          "a batch holds float or double matrices of one kind"));
    }
    SparseBytes mb;
    s = ascb::host::ValidateSparse(m, v.device, &mb);
    if (!s.ok()) return Done(v, s);
    Span xs, ys;
    s = ascb::host::ValidateVector(inputs[i], m.element_kind, false, v.device, &xs);
    if (!s.ok()) return Done(v, s);
    s = ascb::host::ValidateVector(outputs[i], m.element_kind, true, v.device, &ys);
    if (!s.ok()) return Done(v, s);
    if (inputs[i].extent != m.columns || outputs[i].extent != m.rows) {
      return Done(v, Fail(ASC_SB_SHAPE, "batched SpMV vector lengths do not match a matrix"));
    }
    if (ascb::host::Overlap(xs, ys) || ascb::host::Overlap({m.structure_first, mb.first}, ys) ||
        ascb::host::Overlap({m.structure_second, mb.second}, ys) ||
        ascb::host::Overlap({m.values, mb.values}, ys)) {
      return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batched SpMV rejects output operand overlap"));
    }
    writes.push_back(ys);
    reads.push_back(xs);
    reads.push_back({m.structure_first, mb.first});
    reads.push_back({m.structure_second, mb.second});
    reads.push_back({m.values, mb.values});
    ascb_batch_item& it = b->items[static_cast<std::size_t>(i)];
    it.ptr = static_cast<const std::int64_t*>(m.structure_first);
    it.idx = static_cast<const std::int64_t*>(m.structure_second);
    it.val = m.values;
    it.x = inputs[i].data;
    it.y = const_cast<void*>(outputs[i].data);
    it.rows = m.rows;
    it.nnz = m.nonzeros;
    it.incx = inputs[i].stride;
    it.incy = outputs[i].stride;
    it.tile_base = tile_base;
    it.bound_base = tile_base + i;
    tile_base += m.rows > 0 ? Tiles(m.rows, m.nonzeros) : 0;
    b->unit = b->unit && it.incx == 1 && it.incy == 1;
    b->aligned = b->aligned &&
                 ((reinterpret_cast<std::uintptr_t>(it.idx) |
                   reinterpret_cast<std::uintptr_t>(it.val)) &
                  static_cast<std::uintptr_t>(ascb_spmv_seg_alignment() - 1)) == 0;
  }
  if (OutputsOverlap(std::move(writes), reads)) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT,
                        "batched SpMV outputs overlap another output or an input of the batch"));
  }
  if (workspace_bytes < l.total || (l.total != 0 && workspace == nullptr) ||
      (reinterpret_cast<std::uintptr_t>(workspace) & (kAlign - 1)) != 0) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT,
                        "batch workspace is missing, too small or not 256-byte aligned"));
  }
  s = ascb::host::ValidateDevicePointer(workspace, workspace_bytes, v.device,
                                        "CUDA could not inspect batch workspace");
  if (!s.ok()) return Done(v, s);
  auto* ws = static_cast<unsigned char*>(workspace);
  b->items_dev = reinterpret_cast<ascb_batch_item*>(ws + l.items);
  b->bounds = reinterpret_cast<std::int64_t*>(ws + l.bounds);
  b->queue = reinterpret_cast<unsigned long long*>(ws + l.queue);
  b->total_tiles = l.total_tiles;
  b->total_bounds = l.total_bounds;
  if (count > 0) {
    cudaError_t e = cudaMemcpyAsync(b->items_dev, b->items.data(),
                                    b->items.size() * sizeof(ascb_batch_item),
                                    cudaMemcpyHostToDevice, v.stream);
    if (e == cudaSuccess) {
      e = static_cast<cudaError_t>(ascb_batch_tile_bounds(v.stream, b->items_dev, count, b->bounds,
                                                          b->total_bounds, v.sm_count));
      v.launches->fetch_add(1, std::memory_order_relaxed);
    }
    // the host table must outlive the copy: wait for it here (creation is
    // a setup step, not a product)
    const cudaError_t sync = cudaStreamSynchronize(v.stream);
    if (e == cudaSuccess) e = sync;
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return Done(v, {ASC_SB_PROVIDER,
                      std::string("CUDA could not set up the batch: ") + cudaGetErrorString(e)});
    }
  }
  *out = b.release();
  return Done(v, Status::Ok());
}

int asc_sb_batch_destroy(asc_sb_batch* batch) {
  if (batch == nullptr) return ASC_SB_OK;
  DropGraph(batch);
  delete batch;
  return ASC_SB_OK;
}

int asc_sb_batch_set_schedule(asc_sb_context* context, asc_sb_batch* batch, int32_t chunk_tiles,
                              int32_t ctas_per_sm) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (batch == nullptr || chunk_tiles < 1 || chunk_tiles > 4096 || ctas_per_sm < 0 ||
      ctas_per_sm > 32) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch schedule is out of range"));
  }
  batch->chunk = chunk_tiles;
  batch->ctas_per_sm = ctas_per_sm;
  return Done(v, Status::Ok());
}

int asc_sb_batch_get_schedule(const asc_sb_batch* batch, int32_t* chunk_tiles,
                              int32_t* ctas_per_sm) {
  if (batch == nullptr || chunk_tiles == nullptr || ctas_per_sm == nullptr) {
    return ASC_SB_INVALID_ARGUMENT;
  }
  *chunk_tiles = batch->chunk;
  *ctas_per_sm = batch->ctas_per_sm;
  return ASC_SB_OK;
}

int asc_sb_batch_spmv(asc_sb_context* context, asc_sb_batch* batch, double alpha, double beta) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (batch == nullptr) return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "null batch"));
  if (batch->device != v.device) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch and context devices differ"));
  }
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  return Done(v, RunBatch(v, batch, alpha, beta));
}

int asc_sb_batch_spmv_per_matrix(asc_sb_context* context, asc_sb_batch* batch, double alpha,
                                 double beta) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (batch == nullptr) return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "null batch"));
  if (batch->device != v.device) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch and context devices differ"));
  }
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  const int exact = v.determinism == ASC_SB_DETERMINISTIC ? 1 : 0;
  return Done(v, PerMatrix(v, *batch, exact, alpha, beta));
}

int asc_sb_batch_capture(asc_sb_context* context, asc_sb_batch* batch, double alpha,
                         double beta) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (batch == nullptr) return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "null batch"));
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  DropGraph(batch);
  if (!batch->aligned || batch->total_tiles == 0) return Done(v, Status::Ok());
  const int exact = v.determinism == ASC_SB_DETERMINISTIC ? 1 : 0;
  // capture on a private stream: the context stream may be the legacy
  // default stream, which cannot be captured
  cudaStream_t cap = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  cudaGraph_t graph = nullptr;
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const int rc = EnqueuePersistent(cap, *batch, exact, alpha, beta, v.sm_count);
    const cudaError_t end = cudaStreamEndCapture(cap, &graph);
    e = rc != 0 ? static_cast<cudaError_t>(rc) : end;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&batch->exec, graph, 0);
  if (graph != nullptr) (void)cudaGraphDestroy(graph);
  if (cap != nullptr) (void)cudaStreamDestroy(cap);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    DropGraph(batch);
    return Done(v, {ASC_SB_PROVIDER,
                    std::string("CUDA could not capture the batch: ") + cudaGetErrorString(e)});
  }
  batch->g_alpha = alpha;
  batch->g_beta = beta;
  batch->g_exact = exact;
  batch->g_chunk = batch->chunk;
  batch->g_ctas = batch->ctas_per_sm;
  return Done(v, Status::Ok());
}

int asc_sb_batch_autotune(asc_sb_context* context, asc_sb_batch* batch, double alpha,
                          double beta, int32_t reps, float* best_ms) {
  ContextView v;
  if (!ascb::host::ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ascb::host::ViewContext(context, &v);  // determinism and stream as of the lock
  if (batch == nullptr || reps < 1) {
    return Done(v, Fail(ASC_SB_INVALID_ARGUMENT, "batch autotune arguments are invalid"));
  }
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (!batch->aligned || batch->total_tiles == 0) {
    if (best_ms != nullptr) *best_ms = 0.0f;
    return Done(v, Status::Ok());
  }
  const int exact = v.determinism == ASC_SB_DETERMINISTIC ? 1 : 0;
  static const int kChunks[] = {1, 2, 4, 8, 16, 32};
  static const int kCtas[] = {0, 4, 2};
  cudaEvent_t start = nullptr, stop = nullptr;
  cudaError_t e = cudaEventCreate(&start);
  if (e == cudaSuccess) e = cudaEventCreate(&stop);
  float best = -1.0f;
  int best_chunk = batch->chunk, best_ctas = batch->ctas_per_sm;
  for (int chunk : kChunks) {
    for (int ctas : kCtas) {
      if (e != cudaSuccess) break;
      batch->chunk = chunk;
      batch->ctas_per_sm = ctas;
      int rc = EnqueuePersistent(v.stream, *batch, exact, alpha, beta, v.sm_count);  // warm-up
      if (rc == 0) e = cudaEventRecord(start, v.stream);
      for (int r = 0; r < reps && rc == 0 && e == cudaSuccess; ++r) {
        rc = EnqueuePersistent(v.stream, *batch, exact, alpha, beta, v.sm_count);
        v.launches->fetch_add(1, std::memory_order_relaxed);
      }
      if (rc != 0) e = static_cast<cudaError_t>(rc);
      if (e == cudaSuccess) e = cudaEventRecord(stop, v.stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(stop);
      float ms = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, start, stop);
      if (e == cudaSuccess && (best < 0.0f || ms < best)) {
        best = ms;
        best_chunk = chunk;
        best_ctas = ctas;
      }
    }
  }
  if (start != nullptr) (void)cudaEventDestroy(start);
  if (stop != nullptr) (void)cudaEventDestroy(stop);
  batch->chunk = best_chunk;
  batch->ctas_per_sm = best_ctas;
  if (e != cudaSuccess) {
    (void)cudaStreamSynchronize(v.stream);
    (void)cudaGetLastError();
    return Done(v, {ASC_SB_PROVIDER,
                    std::string("CUDA failed while tuning the batch: ") + cudaGetErrorString(e)});
  }
  if (best_ms != nullptr) *best_ms = best / static_cast<float>(reps);
  return Done(v, Status::Ok());
}

}  // extern "C"
