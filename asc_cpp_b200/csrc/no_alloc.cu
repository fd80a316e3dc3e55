// CSR SpMV that allocates nothing: asc_sb_csr_spmv_no_alloc.
//
// Some callers cannot allocate device memory at the point where they need a
// sparse product, and cannot hand in a workspace either: plugin hosts whose
// device memory belongs to the host application's own allocator (which
// forbids raw device allocations by plugins), and latency-critical loops that
// must not take the implicit device synchronisation a cudaMalloc or cudaFree
// may cause.  This entry point serves them: the only scratch memory it needs
// -- the row-tile partition of the matrix -- lives in one file-scope device
// array that every GPU holds from the moment this library is loaded until the
// process exits.
//
// Limits and rules, stated for users:
//   * the array holds kNoAllocMaxBounds int64 tile bounds (2 MiB per GPU); a
//     matrix whose index and value arrays start on 16-byte boundaries needs
//     ceil((2*rows + nnz) / 251) + 1 of them (the segmented kernel's row
//     tiles, as asc_sb_csr_spmv uses), so up to about 65 million weighted
//     items (for example 4 million rows with 57 million nonzeros); other
//     matrices need ceil((8*rows + nnz) / 256) + 1.  Larger matrices are
//     rejected with ASC_SB_UNSUPPORTED and a message naming the limit;
//   * every call on a device shares the one array.  Calls whose work overlaps
//     on the GPU -- two streams, or two contexts on the same device, without
//     ordering between them -- race on it and may compute wrong results;
//   * the array keeps whatever the last call wrote; each call overwrites every
//     entry it reads before reading it, so nothing needs clearing;
//   * it always runs the default kernel (neither a variant forced with
//     asc_sb_context_set_variant nor a selector pick applies): its results
//     equal asc_sb_csr_spmv's bit for bit in DETERMINISTIC mode, and in
//     BACKEND_DEFAULT mode whenever that call also runs the default kernel
//     (both meet the same bound);
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) and keeps it.  Make that first call before any
//     stream capture starts on that device.  A cudaDeviceReset invalidates
//     the kept address: the entry point must not be used after one.
// It calls no cudaMalloc, cudaFree or allocating library routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/asc_sparse_b200.h"
#include "host/context_view.h"
#include "host/validate.h"
#include "kernels.h"

namespace {

constexpr int64_t kNoAllocMaxBounds = int64_t{1} << 18;  // 2 MiB of int64
constexpr int kMaxDevices = 64;

// The scratch array.  Host code must not take its address directly (that is a
// host-side stand-in); it uses the device address found by ScratchFor().
static __device__ __align__(256) int64_t g_tile_bounds[kNoAllocMaxBounds];

std::mutex g_setup_mutex;
int64_t* g_device_address[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
cudaError_t ScratchFor(int device, int64_t** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_device_address[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_tile_bounds);
    if (e != cudaSuccess) return e;
    g_device_address[device] = static_cast<int64_t*>(p);
  }
  *out = g_device_address[device];
  return cudaSuccess;
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

int Done(const ascb::host::ContextView& v, int code, const std::string& message) {
  *v.last_error = code == ASC_SB_OK ? std::string() : message;
  return code;
}

}  // namespace

extern "C" ASC_SB_API int asc_sb_csr_spmv_no_alloc(asc_sb_context* context, double alpha,
                                                   const asc_sb_sparse* matrix,
                                                   const asc_sb_vector* input, double beta,
                                                   const asc_sb_vector* output) {
  using namespace ascb::host;
  ContextView v;
  if (!ViewContext(context, &v)) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(*v.mutex);
  ViewContext(context, &v);  // determinism and stream as of the lock
  Guard guard(v.device);
  if (!guard.ok()) return Done(v, ASC_SB_UNAVAILABLE, "CUDA device is unavailable");
  if (matrix == nullptr || input == nullptr || output == nullptr) {
    return Done(v, ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV descriptors cannot be null");
  }
  if (matrix->format != ASC_SB_CSR) {
    return Done(v, ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV requires CSR format");
  }
  SparseBytes mb;
  Status s = ValidateSparse(*matrix, v.device, &mb);
  if (!s.ok()) return Done(v, s.code, s.message);
  if (matrix->element_kind != ASC_SB_FLOAT && matrix->element_kind != ASC_SB_DOUBLE) {
    return Done(v, ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV supports float and double");
  }
  Span xs, ys;
  s = ValidateVector(*input, matrix->element_kind, false, v.device, &xs);
  if (!s.ok()) return Done(v, s.code, s.message);
  s = ValidateVector(*output, matrix->element_kind, true, v.device, &ys);
  if (!s.ok()) return Done(v, s.code, s.message);
  if (input->extent != matrix->columns || output->extent != matrix->rows) {
    return Done(v, ASC_SB_SHAPE, "CUDA CSR SpMV vector lengths do not match the matrix");
  }
  if (Overlap(xs, ys) || Overlap({matrix->structure_first, mb.first}, ys) ||
      Overlap({matrix->structure_second, mb.second}, ys) || Overlap({matrix->values, mb.values}, ys)) {
    return Done(v, ASC_SB_INVALID_ARGUMENT, "CUDA CSR SpMV rejects output operand overlap");
  }
  if (matrix->rows == 0) return Done(v, ASC_SB_OK, "");

  // the partition asc_sb_csr_spmv uses for the same arrays
  const bool seg_aligned =
      ((reinterpret_cast<std::uintptr_t>(matrix->structure_second) |
        reinterpret_cast<std::uintptr_t>(matrix->values)) &
       static_cast<std::uintptr_t>(ascb_spmv_seg_alignment() - 1)) == 0;
  const int64_t items = seg_aligned ? ascb_seg_tile_items() : ascb_warp_tile_items();
  const int64_t weight = seg_aligned ? ascb_seg_tile_row_weight() : ascb_warp_tile_row_weight();
  const int64_t tiles = ascb_row_tile_count(matrix->rows, matrix->nonzeros, items, weight);
  if (tiles + 1 > kNoAllocMaxBounds) {
    return Done(v, ASC_SB_UNSUPPORTED,
                "matrix too large for the no-allocation SpMV: it needs " +
                    std::to_string(tiles + 1) + " tile bounds, the static scratch holds " +
                    std::to_string(kNoAllocMaxBounds));
  }
  int64_t* scratch = nullptr;
  cudaError_t e = ScratchFor(v.device, &scratch);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return Done(v, ASC_SB_PROVIDER,
                std::string("could not locate the static scratch: ") + cudaGetErrorString(e));
  }

  ascb_csr a{};
  a.rows = matrix->rows;
  a.cols = matrix->columns;
  a.nnz = matrix->nonzeros;
  a.ptr = static_cast<const int64_t*>(matrix->structure_first);
  a.idx = static_cast<const int64_t*>(matrix->structure_second);
  a.val = matrix->values;
  const ascb_vec xv{const_cast<void*>(input->data), input->extent, input->stride};
  const ascb_vec yv{const_cast<void*>(output->data), output->extent, output->stride};
  const int dtype = matrix->element_kind == ASC_SB_DOUBLE ? ASCB_F64 : ASCB_F32;
  const int exact = v.determinism == ASC_SB_DETERMINISTIC ? 1 : 0;

  int rc = ascb_row_tiles(v.stream, &a, items, weight, scratch, tiles);
  v.launches->fetch_add(1, std::memory_order_relaxed);
  if (rc == 0) {
    rc = seg_aligned ? ascb_spmv_seg_w(v.stream, dtype, ASCB_COMPAT, exact, &a, alpha, beta, &xv,
                                       &yv, scratch, tiles, weight, v.sm_count)
                   : ascb_spmv_warp(v.stream, dtype, ASCB_COMPAT, exact, &a, alpha, beta, &xv, &yv,
                                    scratch, tiles, v.sm_count);
    v.launches->fetch_add(1, std::memory_order_relaxed);
  }
  if (rc != 0) {
    (void)cudaStreamSynchronize(v.stream);
    (void)cudaGetLastError();
    return Done(v, ASC_SB_PROVIDER,
                std::string("CUDA could not launch the no-allocation SpMV: ") +
                    cudaGetErrorString(static_cast<cudaError_t>(rc)));
  }
  return Done(v, ASC_SB_OK, "");
}
