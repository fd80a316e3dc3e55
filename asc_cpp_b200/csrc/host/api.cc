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
#include <vector>

#include "../../../include/asc_sparse_b200.h"
#include "../kernels.h"
#include "context_view.h"
#include "memory.h"
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
  std::uint64_t wait_ns = 0;  // dependency-wait limit of solves (0: the kernels' 2 s)
  void* scratch = nullptr;  // kContextScratch device bytes after the status word
  // installed variant selector: device parameters and scratch, and the
  // variant (id, lanes) each MLP output stands for
  int selector_outputs = 0;
  float* selector = nullptr;
  std::vector<int> selector_variant, selector_lanes;
  // triangular solves without a plan: ready flags (and, for transposed
  // solves, the transposed structure) in a buffer that grows to the largest
  // solve seen
  ascb::host::Block solve_mem;
  ascb::host::Block selector_mem;  // holds `selector`
  ascb::host::Allocator allocator;  // for the blocks above and clone staging
  // selector picks of matrices used without a plan (ChooseWithoutPlan)
  struct PickKey {
    const void* ptr = nullptr;
    const void* idx = nullptr;
    const void* val = nullptr;
    std::int64_t rows = 0, cols = 0, nnz = 0;
    std::int32_t kind = 0, format = 0;
    bool operator==(const PickKey&) const = default;
  };
  struct PickSlot {
    PickKey key;
    int state = 0;  // 0 empty, 1 selection in flight, 2 pick ready
    int pick = -1;
    std::uint64_t used = 0;
    cudaEvent_t done = nullptr;
  };
  static constexpr int kPickSlots = 16;
  PickSlot picks[kPickSlots];
  ascb::host::Block pick_words;  // pinned host: one int per slot
  int pick_in_flight = -1;
  std::uint64_t pick_clock = 0;
  void* stager = nullptr;  // clone staging, clone.cc
};

constexpr std::size_t kContextScratchOffset = 256;
constexpr std::size_t kContextScratch = 4096;

// Partitions of one CSR structure, as the kernels consume them.
struct Partitions {
  const std::int64_t* warp_tiles = nullptr;    // ascb_row_tiles, warp-tile weights
  std::int64_t n_warp = 0;
  void* split = nullptr;  // row-split block (ascb_split_bytes(nnz, 256) bytes)
  const std::int64_t* seg_tiles = nullptr;  // the segmented kernel's own row tiles
  std::int64_t n_seg = 0;
  const std::int64_t* merge_tiles = nullptr;  // the merge partition's row tiles (weight 1)
  std::int64_t n_merge_tiles = 0;
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
  // variant picked for this matrix (selector or exhaustive autotune);
  // variant < -1 means none
  int variant = -2;
  int lanes = 0;
  // FP32 CSR made of dense, aligned 16 x 16 blocks: SpMM runs on the tensor
  // cores in BACKEND_DEFAULT mode
  bool block16 = false;
  // ASC_SB_PLAN_TRIANGULAR: control block and published values of the
  // solves, and room for one level analysis (asc_sb_plan_triangular_analysis)
  unsigned char* solve = nullptr;
  unsigned char* analysis = nullptr;
  bool analysed = false;
  bool analysis_transposed = false;  // analysis of op != none
  bool analysis_lower = false;       // of a lower triangular op(A)
  const std::int64_t* order = nullptr;
  const std::int64_t* position = nullptr;
  // ASC_SB_PLAN_ROW_GROUPS: runs of R consecutive rows for the row-group SpMM
  unsigned char* groups_mem = nullptr;
  ascb_row_groups groups{};
  std::int64_t group_run_count = 0;
  bool use_groups = false;  // SpMM through the groups (reuse measured or tuned)
  // ASC_SB_PLAN_ROW_GROUPS also builds the TMA-staged SpMM tables (groups of
  // 16 rows, and wide groups of 32 and 64 whose shared columns are one slot);
  // staged_caps[v][2w], [2w + 1]: largest slot and entry counts of a stage
  // of 2^w groups of level v
  unsigned char* staged_mem = nullptr;
  ascb_staged_spmm staged[ASCB_STAGED_LEVELS] = {};
  std::int64_t staged_caps[ASCB_STAGED_LEVELS][10] = {};
  bool level_ok[ASCB_STAGED_LEVELS] = {};  // no group of the level exceeds 65534 slots
  std::int64_t staged_slots = 0;  // distinct columns over all 16-row groups
  bool has_staged = false;
  bool use_staged = false;    // SpMM through the staged kernel where it fits ...
  bool staged_tuned = false;  // ... for every k (the autotuner picked it), else for k >= 8
  // the last SpMM autotune: candidates timed and their ms per product
  int tuned_count = 0;
  int tuned_candidate[8] = {};
  float tuned_ms[8] = {};
};

namespace {

#include "selector_default.inc"

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
// Result of an enqueue of `kernels` kernels (counted in the context's launch
// counter).
Status Launched(asc_sb_context* ctx, int err, const char* message, int kernels = 1) {
  ctx->launches.fetch_add(kernels, std::memory_order_relaxed);
  if (err == 0) return Status::Ok();
  (void)cudaStreamSynchronize(ctx->stream);
  (void)cudaGetLastError();
  return {ASC_SB_PROVIDER,
          std::string(message) + ": " + cudaGetErrorString(static_cast<cudaError_t>(err))};
}

bool RealKind(int kind) { return kind == ASC_SB_FLOAT || kind == ASC_SB_DOUBLE; }

int Dtype(int kind) {
  switch (kind) {
    case ASC_SB_DOUBLE: return ASCB_F64;
    case ASC_SB_COMPLEX_FLOAT: return ASCB_C64;
    case ASC_SB_COMPLEX_DOUBLE: return ASCB_C128;
    default: return ASCB_F32;
  }
}

// alpha == 0 in the element type: real kinds take the real part only, as the
// reference's ScalarValue conversion does (kernels.cu:15-17, 45-47).
bool AlphaIsZero(int kind, double alpha_real, double alpha_imag) {
  return RealKind(kind) ? alpha_real == 0.0 : (alpha_real == 0.0 && alpha_imag == 0.0);
}

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
std::int64_t SegTiles(std::int64_t rows, std::int64_t nnz) {
  return ascb_row_tile_count(rows, nnz, ascb_seg_tile_items(), ascb_seg_tile_row_weight());
}
std::size_t SegTileBytes(std::int64_t rows, std::int64_t nnz) {
  return RoundUp(static_cast<std::size_t>(SegTiles(rows, nnz) + 1) * 8, 256);
}
std::int64_t MergeTiles(std::int64_t rows, std::int64_t nnz) {
  return ascb_row_tile_count(rows, nnz, ascb_merge_tile_items(), ascb_merge_tile_row_weight());
}
std::size_t MergeTileBytes(std::int64_t rows, std::int64_t nnz) {
  return RoundUp(static_cast<std::size_t>(MergeTiles(rows, nnz) + 1) * 8, 256);
}
// Room for any row-tile partition (the segmented kernel's has fewer tiles
// unless rows average more than about 300 entries).
std::size_t TileBytes(std::int64_t rows, std::int64_t nnz) {
  return std::max({WarpTileBytes(rows, nnz), SegTileBytes(rows, nnz), MergeTileBytes(rows, nnz)});
}

// ---- workspace layout of asc_sb_csr_spmv ----------------------------------
// The size is a function of the matrix shape only, so it is stable for a given
// (A, x, y) (the reference's rule, operations.cc:884-909): room for the
// partition of whichever kernel the context selects.
// Row-split block of a structure with `nnz` entries, sized for the smallest
// split threshold (tails longer than 256 positions), so one block serves
// every threshold.
std::size_t SplitBlockBytes(std::int64_t nnz) {
  return RoundUp(ascb_split_bytes(nnz, 256), 256);
}
std::size_t CompatWorkspaceBytes(const asc_sb_sparse& m) {
  if (m.rows == 0 || m.columns == 0) return 0;
  return TileBytes(m.rows, m.nonzeros) + SplitBlockBytes(m.nonzeros);
}

// ROW_SPLIT: a row is split when its tail past the tile window exceeds this
// many 256-position rounds (the context's or plan's "lanes" value overrides).
constexpr std::int64_t kSplitRounds = 4;

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

// Variant for a real CSR product: DETERMINISTIC always takes the bit-exact
// row-ordered kernels; otherwise a variant forced on the context, else the
// plan's pick (selector or autotune), else the default, WARP_TILES.
Choice Choose(const asc_sb_context* ctx, const asc_sb_sparse& m, int plan_variant = -2,
              int plan_lanes = 0) {
  Choice c;
  if (ctx->determinism == ASC_SB_DETERMINISTIC) return c;  // bit-exact order
  if (ctx->variant != ASC_SB_VARIANT_AUTO) {
    c.variant = ctx->variant;
    c.lanes = ctx->lanes > 0 ? ctx->lanes : AutoLanes(m, false);
    return c;
  }
  if (plan_variant >= 0) {
    c.variant = plan_variant;
    c.lanes = plan_lanes > 0 ? plan_lanes : AutoLanes(m, false);
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
  // The register-segmented kernel needs 16-byte aligned index and value
  // arrays; otherwise every variant but VECTOR runs the scalar-load warp
  // kernel.
  const bool seg_aligned =
      ((reinterpret_cast<std::uintptr_t>(a.idx) | reinterpret_cast<std::uintptr_t>(a.val)) &
       static_cast<std::uintptr_t>(ascb_spmv_seg_alignment() - 1)) == 0;
  if (choice.variant == ASC_SB_VARIANT_MERGE_PATH && seg_aligned) {
    // the merge partition -- equal shares of rows plus nonzeros, one item
    // each -- run by the segmented kernel's tile body (up to 250 rows a tile)
    const std::int64_t weight = ascb_merge_tile_row_weight();
    const std::int64_t items = ascb_merge_tile_items();
    const std::int64_t tiles = ascb_row_tile_count(a.rows, a.nnz, items, weight);
    const std::int64_t* tiles_ptr = planned != nullptr ? planned->merge_tiles : nullptr;
    if (tiles_ptr == nullptr && scratch != nullptr) {
      Status s = Launched(ctx, ascb_row_tiles(ctx->stream, &a, items, weight, scratch, tiles),
                          "CUDA could not launch the row-tile partition kernel");
      if (!s.ok()) return s;
      tiles_ptr = scratch;
    }
    return Launched(ctx,
                    ascb_spmv_seg_w(ctx->stream, dtype, form, 0, &a, alpha, beta, &x, &y,
                                    tiles_ptr, tiles, weight, ctx->sm_count),
                    "CUDA could not launch the segmented SpMV kernel");
  }
  // ROW_ORDERED (bit-exact) and WARP_TILES (contracted) run the register-
  // segmented kernel on its own row tiles (up to 125 rows each) when the
  // arrays are aligned; otherwise the scalar-load warp kernel, with the same
  // numerics, on tiles of at most 32 rows.  Any partition fits the front of
  // the workspace.
  const std::int64_t weight =
      seg_aligned ? ascb_seg_tile_row_weight() : ascb_warp_tile_row_weight();
  const std::int64_t items = seg_aligned ? ascb_seg_tile_items() : ascb_warp_tile_items();
  const std::int64_t tiles = ascb_row_tile_count(a.rows, a.nnz, items, weight);
  const std::int64_t* tiles_ptr =
      planned != nullptr ? (seg_aligned ? planned->seg_tiles : planned->warp_tiles) : nullptr;
  if (tiles_ptr == nullptr && scratch != nullptr) {
    Status s = Launched(ctx,
                        ascb_row_tiles(ctx->stream, &a, items, weight, scratch, tiles),
                        "CUDA could not launch the row-tile partition kernel");
    if (!s.ok()) return s;
    tiles_ptr = scratch;
  }
  if (choice.variant == ASC_SB_VARIANT_ROW_SPLIT && seg_aligned) {
    // the split block lives in the plan, or after the tile bounds in the
    // caller's workspace; without either (the standard path without a plan)
    // the row runs inline, as in WARP_TILES
    void* block = planned != nullptr ? planned->split
                  : scratch != nullptr
                      ? static_cast<void*>(reinterpret_cast<unsigned char*>(scratch) +
                                           TileBytes(a.rows, a.nnz))
                      : nullptr;
    if (block != nullptr) {
      const std::int64_t rounds = choice.lanes > 0 ? choice.lanes : kSplitRounds;
      return Launched(ctx,
                      ascb_spmv_split(ctx->stream, dtype, form, &a, alpha, beta, &x, &y,
                                      tiles_ptr, tiles, weight, rounds * ascb_warp_tile_items(),
                                      block, ctx->sm_count),
                      "CUDA could not launch the row-split SpMV kernels", 2);
    }
  }
  if (seg_aligned) {
    return Launched(ctx,
                    ascb_spmv_seg_w(ctx->stream, dtype, form, exact, &a, alpha, beta, &x, &y,
                                    tiles_ptr, tiles, weight, ctx->sm_count),
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
  auto* warp = reinterpret_cast<std::int64_t*>(buffer);
  out->warp_tiles = warp;
  out->split = buffer + WarpTileBytes(a.rows, a.nnz);
  auto* seg = reinterpret_cast<std::int64_t*>(static_cast<unsigned char*>(out->split) +
                                              SplitBlockBytes(a.nnz));
  out->seg_tiles = seg;
  out->n_seg = SegTiles(a.rows, a.nnz);
  auto* mtiles = reinterpret_cast<std::int64_t*>(reinterpret_cast<unsigned char*>(seg) +
                                                 SegTileBytes(a.rows, a.nnz));
  out->merge_tiles = mtiles;
  out->n_merge_tiles = MergeTiles(a.rows, a.nnz);
  if (a.rows == 0) return Status::Ok();
  Status s = Launched(ctx,
                      ascb_row_tiles(ctx->stream, &a, ascb_warp_tile_items(),
                                     ascb_warp_tile_row_weight(), warp, out->n_warp),
                      "CUDA could not launch the row-tile partition kernel");
  if (!s.ok()) return s;
  s = Launched(ctx,
               ascb_row_tiles(ctx->stream, &a, ascb_seg_tile_items(), ascb_seg_tile_row_weight(),
                              seg, out->n_seg),
               "CUDA could not launch the row-tile partition kernel");
  if (!s.ok()) return s;
  return Launched(ctx,
                  ascb_row_tiles(ctx->stream, &a, ascb_merge_tile_items(),
                                 ascb_merge_tile_row_weight(), mtiles, out->n_merge_tiles),
                  "CUDA could not launch the row-tile partition kernel");
}
std::size_t PartitionBytes(std::int64_t rows, std::int64_t nnz) {
  return WarpTileBytes(rows, nnz) + SplitBlockBytes(nnz) + SegTileBytes(rows, nnz) +
         MergeTileBytes(rows, nnz);
}

std::size_t EntryBytes(std::int64_t nnz, std::size_t element) {
  return RoundUp(static_cast<std::size_t>(nnz > 0 ? nnz : 1) * element, 256);
}

// Layout of a plan's workspace.  Without ASC_SB_PLAN_TRANSPOSE it holds the
// partitions of the stored arrays only.  With it, also the transposed
// structure (offsets, indices, the permutation that maps its entries to the
// stored ones, and its values), that structure's partitions, and the scratch
// the stable sort uses while the plan is created.
struct PlanLayout {
  std::size_t flag = 0;  // one device int for structure checks
  std::size_t t_ptr = 0, t_idx = 0, t_perm = 0, t_val = 0, t_part = 0;
  std::size_t sort = 0, outer_of = 0, solve = 0, analysis = 0, groups = 0, staged = 0, total = 0;
};

PlanLayout PlanLayoutFor(const asc_sb_sparse& m, int flags) {
  const bool csc = m.format == ASC_SB_CSC;
  const std::int64_t outer = csc ? m.columns : m.rows;
  const std::int64_t inner = csc ? m.rows : m.columns;
  const std::int64_t nnz = m.nonzeros;
  PlanLayout l;
  std::size_t at = PartitionBytes(outer, nnz);
  l.flag = at;
  at += 256;
  if (flags & ASC_SB_PLAN_TRANSPOSE) {
    l.t_ptr = at;
    at += RoundUp(static_cast<std::size_t>(inner + 1) * 8, 256);
    l.t_idx = at;
    at += EntryBytes(nnz, 8);
    l.t_perm = at;
    at += EntryBytes(nnz, 8);
    l.t_val = at;
    at += EntryBytes(nnz, ascb::host::ElementBytes(m.element_kind));
    l.t_part = at;
    at += PartitionBytes(inner, nnz);
    l.sort = at;
    at += RoundUp(ascb_sort_workspace_bytes(nnz, inner), 256);
    l.outer_of = at;
    at += EntryBytes(nnz, 8);
  }
  if (flags & ASC_SB_PLAN_TRIANGULAR) {
    l.solve = at;
    at += RoundUp(ascb_trsv_scratch_bytes(
                      outer, static_cast<int>(ascb::host::ElementBytes(m.element_kind))),
                  256);
    l.analysis = at;
    at += RoundUp(ascb_trsv_analysis_bytes(outer), 256);
  }
  if (flags & ASC_SB_PLAN_ROW_GROUPS) {
    l.groups = at;
    at += RoundUp(ascb_row_groups_layout_for(
                      outer, nnz, static_cast<int>(ascb::host::ElementBytes(m.element_kind)))
                      .total,
                  256);
    l.staged = at;
    at += RoundUp(ascb_staged_layout_for(outer, nnz).total, 256);
  }
  l.total = at;
  return l;
}

// Row groups of R rows for the plan's CSR arrays; reads back the number of
// runs (synchronizes the stream) and keeps the groups in use when they share
// B rows: at least 1.25 stored entries per run.
constexpr int kDefaultRowsPerGroup = 8;
Status BuildRowGroups(asc_sb_context* ctx, asc_sb_plan* plan, int rows_per_group) {
  const ascb_csr a = AsCsr(plan->matrix, false);
  const int elem = static_cast<int>(ascb::host::ElementBytes(plan->matrix.element_kind));
  Status s = Launched(ctx,
                      ascb_row_groups_build(ctx->stream, &a, elem, rows_per_group,
                                            plan->groups_mem, &plan->groups, ctx->sm_count),
                      "CUDA could not launch the row-group build");
  if (!s.ok()) return s;
  const std::int64_t groups = (a.rows + rows_per_group - 1) / rows_per_group;
  std::int64_t runs = 0;
  cudaError_t e = cudaMemcpyAsync(&runs, plan->groups.group_runs + groups, sizeof(runs),
                                  cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return {ASC_SB_PROVIDER, std::string("CUDA could not build the row groups: ") +
                                 cudaGetErrorString(e)};
  }
  plan->group_run_count = runs;
  plan->use_groups = runs > 0 && 4 * a.nnz >= 5 * runs;
  return Status::Ok();
}

// The TMA-staged SpMM tables, from row groups of 16 rows built just before
// (their build scratch is read); reads back the stage caps (synchronizes the
// stream).  Used by default when the groups share columns (at least 1.25
// stored entries per distinct column of a group).
Status BuildStaged(asc_sb_context* ctx, asc_sb_plan* plan) {
  const ascb_csr a = AsCsr(plan->matrix, false);
  const int elem = static_cast<int>(ascb::host::ElementBytes(plan->matrix.element_kind));
  Status s = Launched(ctx,
                      ascb_staged_build(ctx->stream, &a, &plan->groups, plan->groups_mem, elem,
                                        plan->staged_mem, plan->staged, ctx->sm_count),
                      "CUDA could not launch the staged SpMM build");
  if (!s.ok()) return s;
  unsigned long long caps[ASCB_STAGED_LEVELS][10] = {};
  cudaError_t e = cudaSuccess;
  for (int v = 0; v < ASCB_STAGED_LEVELS && e == cudaSuccess; ++v) {
    e = cudaMemcpyAsync(caps[v], plan->staged[v].caps, sizeof(caps[v]), cudaMemcpyDeviceToHost,
                        ctx->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return {ASC_SB_PROVIDER, std::string("CUDA could not build the staged SpMM tables: ") +
                                 cudaGetErrorString(e)};
  }
  for (int v = 0; v < ASCB_STAGED_LEVELS; ++v) {
    for (int i = 0; i < 10; ++i) plan->staged_caps[v][i] = static_cast<std::int64_t>(caps[v][i]);
    plan->level_ok[v] = plan->staged_caps[v][0] < 65535;
  }
  plan->has_staged = true;
  const std::int64_t slots = plan->group_run_count;  // of the 16-row groups
  plan->staged_slots = slots;
  plan->use_staged = slots > 0 && 4 * a.nnz >= 5 * slots;
  return Status::Ok();
}

// Stable transposed structure of the CSR arrays `a` (rows = stored outer
// extent): t_ptr [a.cols + 1], t_idx / t_perm / t_val [nnz].
Status BuildTransposed(asc_sb_context* ctx, const ascb_csr& a, std::size_t element,
                       std::int64_t* t_ptr, std::int64_t* t_idx, std::int64_t* t_perm,
                       void* t_val, void* sort_scratch, std::int64_t* outer_of) {
  Status s = Launched(ctx,
                      ascb_stable_sort(ctx->stream, a.idx, 1, a.nnz, a.cols, t_ptr, t_perm,
                                       sort_scratch),
                      "CUDA could not launch the transposition sort");
  if (!s.ok()) return s;
  s = Launched(ctx, ascb_outer_of_entries(ctx->stream, a.ptr, a.rows, outer_of, ctx->sm_count),
               "CUDA could not launch the row expansion kernel");
  if (!s.ok()) return s;
  return Launched(ctx,
                  ascb_permute_entries(ctx->stream, t_perm, a.nnz, outer_of, 1, t_idx, a.val,
                                       t_val, static_cast<int>(element), ctx->sm_count),
                  "CUDA could not launch the entry permutation kernel");
}

// ---- variant selector ------------------------------------------------------
// Device layout of an installed selector (floats): accumulators [0, 16),
// features [16, 28), hidden units [32, 160), outputs [160, 224), the pick
// (an int) at 224, parameters from 256 on.
constexpr int kSelAcc = 0, kSelFeatures = 16, kSelHidden = 32, kSelOut = 160, kSelPick = 224,
              kSelParams = 256, kSelMaxOutputs = 64;

// Runs features -> MLP -> argmin for the plan's matrix and records the
// variant the selector's best output stands for.  Synchronizes the stream.
Status SelectVariant(asc_sb_context* ctx, asc_sb_plan* plan) {
  float* base = ctx->selector;
  const ascb_csr a = AsCsr(plan->matrix, plan->matrix.format == ASC_SB_CSC);
  int rc = ascb_matrix_features(
      ctx->stream, &a, static_cast<int>(ascb::host::ElementBytes(plan->matrix.element_kind)),
      reinterpret_cast<unsigned long long*>(base + kSelAcc), base + kSelFeatures, ctx->sm_count);
  if (rc == 0) {
    rc = ascb_mlp_forward(ctx->stream, ctx->selector_outputs, base + kSelParams,
                          base + kSelFeatures, 1, base + kSelHidden, base + kSelOut);
  }
  if (rc == 0) {
    rc = ascb_argmin(ctx->stream, base + kSelOut, ctx->selector_outputs,
                     reinterpret_cast<int*>(base + kSelPick));
  }
  ctx->launches.fetch_add(6, std::memory_order_relaxed);
  int pick = 0;
  cudaError_t e = static_cast<cudaError_t>(rc);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&pick, base + kSelPick, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  }
  const cudaError_t sync = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = sync;
  if (e != cudaSuccess || pick < 0 || pick >= ctx->selector_outputs) {
    (void)cudaGetLastError();
    return {ASC_SB_PROVIDER, std::string("CUDA could not run the variant selector: ") +
                                 cudaGetErrorString(e)};
  }
  plan->variant = ctx->selector_variant[static_cast<std::size_t>(pick)];
  plan->lanes = ctx->selector_lanes[static_cast<std::size_t>(pick)];
  return Status::Ok();
}

// Variant of a real, non-transposed product without a plan.  With a selector
// installed (BACKEND_DEFAULT, variant AUTO) the first call on a matrix --
// keyed by its arrays and shape -- enqueues the selection (features -> MLP ->
// argmin -> a pinned host word, then an event) ahead of its own product, which
// runs the default; later calls use the pick once the event has completed.  No
// host wait, and nothing is enqueued while the stream is being captured.  A
// stale key (arrays freed and reused for another matrix of the same shape)
// only costs speed: every variant meets the same bound.
Choice ChooseWithoutPlan(asc_sb_context* ctx, const asc_sb_sparse& m) {
  Choice c = Choose(ctx, m);
  if (ctx->determinism == ASC_SB_DETERMINISTIC || ctx->variant != ASC_SB_VARIANT_AUTO ||
      ctx->selector == nullptr || !RealKind(m.element_kind) || m.nonzeros == 0) {
    return c;
  }
  auto& slots = ctx->picks;
  const int* words = static_cast<const int*>(ctx->pick_words.ptr);
  if (ctx->pick_in_flight >= 0) {  // has the selection in flight landed?
    auto& f = slots[ctx->pick_in_flight];
    const cudaError_t q = cudaEventQuery(f.done);
    if (q == cudaSuccess) {
      const int pick = words[ctx->pick_in_flight];
      f.state = pick >= 0 && pick < ctx->selector_outputs ? 2 : 0;
      f.pick = pick;
      ctx->pick_in_flight = -1;
    } else if (q != cudaErrorNotReady) {
      (void)cudaGetLastError();
      f.state = 0;
      ctx->pick_in_flight = -1;
    }
  }
  asc_sb_context::PickKey key{m.structure_first, m.structure_second, m.values, m.rows,
                              m.columns, m.nonzeros, m.element_kind, m.format};
  int victim = -1;
  for (int i = 0; i < asc_sb_context::kPickSlots; ++i) {
    auto& slot = slots[i];
    if (slot.state != 0 && slot.key == key) {
      slot.used = ++ctx->pick_clock;
      if (slot.state == 2) {
        c.variant = ctx->selector_variant[static_cast<std::size_t>(slot.pick)];
        const int lanes = ctx->selector_lanes[static_cast<std::size_t>(slot.pick)];
        c.lanes = lanes > 0 ? lanes : AutoLanes(m, false);
      }
      return c;
    }
    if (slot.state != 1 && (victim < 0 || slot.state == 0 ||
                            (slots[victim].state != 0 && slot.used < slots[victim].used))) {
      victim = i;
    }
  }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (ctx->pick_in_flight >= 0 || victim < 0 ||
      cudaStreamIsCapturing(ctx->stream, &capture) != cudaSuccess ||
      capture != cudaStreamCaptureStatusNone) {
    (void)cudaGetLastError();
    return c;
  }
  if (ctx->pick_words.ptr == nullptr &&
      !ascb::host::Acquire(ctx->allocator, sizeof(int) * asc_sb_context::kPickSlots,
                           ASC_SB_PINNED_HOST, &ctx->pick_words)) {
    return c;  // no room for the answers: keep the default
  }
  auto& slot = slots[victim];
  if (slot.done == nullptr &&
      cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    slot.done = nullptr;
    return c;
  }
  float* base = ctx->selector;
  const ascb_csr a = AsCsr(m, m.format == ASC_SB_CSC);
  int* word = static_cast<int*>(ctx->pick_words.ptr) + victim;
  int rc = ascb_matrix_features(
      ctx->stream, &a, static_cast<int>(ascb::host::ElementBytes(m.element_kind)),
      reinterpret_cast<unsigned long long*>(base + kSelAcc), base + kSelFeatures, ctx->sm_count);
  if (rc == 0) {
    rc = ascb_mlp_forward(ctx->stream, ctx->selector_outputs, base + kSelParams,
                          base + kSelFeatures, 1, base + kSelHidden, base + kSelOut);
  }
  if (rc == 0) {
    rc = ascb_argmin(ctx->stream, base + kSelOut, ctx->selector_outputs,
                     reinterpret_cast<int*>(base + kSelPick));
  }
  ctx->launches.fetch_add(6, std::memory_order_relaxed);
  if (rc == 0) {
    rc = static_cast<int>(cudaMemcpyAsync(word, base + kSelPick, sizeof(int),
                                          cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (rc == 0) rc = static_cast<int>(cudaEventRecord(slot.done, ctx->stream));
  if (rc != 0) {
    (void)cudaGetLastError();
    slot.state = 0;
    return c;
  }
  slot.key = key;
  slot.state = 1;
  slot.pick = -1;
  slot.used = ++ctx->pick_clock;
  ctx->pick_in_flight = victim;
  return c;
}

// Forgets every pick (a new selector was installed); the stream is idle.
void ForgetPicks(asc_sb_context* ctx) {
  for (auto& slot : ctx->picks) {
    slot.state = 0;
    slot.pick = -1;
  }
  ctx->pick_in_flight = -1;
}

// Marks the plan when its matrix is made of dense 16 x 16 blocks (one check
// kernel, then a read of its flag; synchronizes the stream).
Status DetectBlocks(asc_sb_context* ctx, const ascb_csr& a, int* flag, asc_sb_plan* plan) {
  int bad = 1;
  cudaError_t e =
      static_cast<cudaError_t>(ascb_block16_check(ctx->stream, &a, flag, ctx->sm_count));
  ctx->launches.fetch_add(1, std::memory_order_relaxed);
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  }
  const cudaError_t sync = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = sync;
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return {ASC_SB_PROVIDER,
            std::string("CUDA could not check the block structure: ") + cudaGetErrorString(e)};
  }
  plan->block16 = bad == 0;
  return Status::Ok();
}

bool ValidVariant(int variant, int lanes) {
  if (variant == ASC_SB_VARIANT_VECTOR) {
    return lanes >= 1 && lanes <= 32 && (lanes & (lanes - 1)) == 0;
  }
  return variant == ASC_SB_VARIANT_ROW_ORDERED || variant == ASC_SB_VARIANT_WARP_TILES ||
         variant == ASC_SB_VARIANT_MERGE_PATH || variant == ASC_SB_VARIANT_ROW_SPLIT;
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
  // One device word per context for kernels' bounded-wait timeouts and a
  // small scratch (reduction partials) behind it: a set-up allocation, no
  // operation allocates.
  if (cudaMalloc(reinterpret_cast<void**>(&ctx->status), kContextScratchOffset + kContextScratch) !=
          cudaSuccess ||
      cudaMemset(ctx->status, 0, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    if (ctx->owns_stream) (void)cudaStreamDestroy(ctx->stream);
    if (ctx->status != nullptr) (void)cudaFree(ctx->status);
    delete ctx;
    return ASC_SB_ALLOCATION;
  }
  ctx->scratch = reinterpret_cast<unsigned char*>(ctx->status) + kContextScratchOffset;
  // the shipped selector: BACKEND_DEFAULT products with variant AUTO pick
  // their kernel from the start; a context that cannot hold it still works
  // and runs the default variant
  if (asc_sb_context_set_selector(ctx, kDefaultSelectorOutputs, kDefaultSelectorParams,
                                  kDefaultSelectorVariants, kDefaultSelectorLanes) != ASC_SB_OK) {
    ctx->last_error.clear();
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
  for (auto& slot : ctx->picks) {
    if (slot.done != nullptr) (void)cudaEventDestroy(slot.done);
  }
  ascb::host::Release(&ctx->pick_words);
  ascb::host::Release(&ctx->selector_mem);
  ascb::host::Release(&ctx->solve_mem);
  ascb::host::DestroyStager(ctx->stager);
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
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->variant = variant;
  ctx->lanes = lanes;
  return ASC_SB_OK;
}

int asc_sb_context_set_allocator(asc_sb_context* ctx, asc_sb_allocate_fn allocate,
                                 asc_sb_deallocate_fn release, void* user) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->allocator = allocate != nullptr ? ascb::host::Allocator{allocate, release, user}
                                       : ascb::host::Allocator{};
  return ASC_SB_OK;
}

int asc_sb_context_set_wait_limit(asc_sb_context* ctx, int64_t nanoseconds) {
  if (ctx == nullptr) return ASC_SB_INVALID_STATE;
  if (nanoseconds < 0) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "The wait limit cannot be negative"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->wait_ns = static_cast<std::uint64_t>(nanoseconds);
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
  const Choice choice = ChooseWithoutPlan(ctx, *m);
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

Status ValidateStandardSpmv(asc_sb_context* ctx, int op, const asc_sb_sparse* m, const asc_sb_vector* x,
                            const asc_sb_vector* y, StandardOperands* out) {
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid");
  }
  if (m == nullptr || x == nullptr || y == nullptr) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA standardized SpMV descriptors cannot be null");
  }
  Status s = ascb::host::ValidateSparse(*m, ctx->device, &out->matrix_bytes);
  if (!s.ok()) return s;
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

// The plan's transposed structure as CSR arrays (rows = stored inner extent).
ascb_csr TransposedCsr(const asc_sb_plan& plan) {
  const ascb_csr a = AsCsr(plan.matrix, plan.matrix.format == ASC_SB_CSC);
  ascb_csr t{};
  t.rows = a.cols;
  t.cols = a.rows;
  t.nnz = a.nnz;
  t.ptr = plan.t_ptr;
  t.idx = plan.t_idx;
  t.val = plan.t_val;
  return t;
}

Status SolveScratch(asc_sb_context* ctx, std::size_t bytes, unsigned char** out);

// The transposed structure of the CSR arrays `a`, built on the stream into the
// context's scratch buffer (which grows, after a stream drain, to the largest
// request): the deterministic transposed products of callers without a plan.
// Stable by source row, so a stored-order kernel on it adds each output's
// terms in the reference's order (blas.h:1241-1256).
Status TransposedInScratch(asc_sb_context* ctx, const ascb_csr& a, std::size_t element,
                           ascb_csr* out) {
  const std::int64_t nnz = a.nnz;
  std::size_t total = 0;
  const std::size_t t_ptr = total;
  total += RoundUp(static_cast<std::size_t>(a.cols + 1) * 8, 256);
  const std::size_t t_idx = total;
  total += EntryBytes(nnz, 8);
  const std::size_t t_perm = total;
  total += EntryBytes(nnz, 8);
  const std::size_t t_val = total;
  total += EntryBytes(nnz, element);
  const std::size_t sort = total;
  total += RoundUp(ascb_sort_workspace_bytes(nnz, a.cols), 256);
  const std::size_t outer_of = total;
  total += EntryBytes(nnz, 8);
  unsigned char* base = nullptr;
  Status s = SolveScratch(ctx, total, &base);
  if (!s.ok()) return s;
  auto* tp = reinterpret_cast<std::int64_t*>(base + t_ptr);
  auto* ti = reinterpret_cast<std::int64_t*>(base + t_idx);
  s = BuildTransposed(ctx, a, element, tp, ti, reinterpret_cast<std::int64_t*>(base + t_perm),
                      base + t_val, base + sort, reinterpret_cast<std::int64_t*>(base + outer_of));
  if (!s.ok()) return s;
  *out = ascb_csr{};
  out->rows = a.cols;
  out->cols = a.rows;
  out->nnz = a.nnz;
  out->ptr = tp;
  out->idx = ti;
  out->val = base + t_val;
  return Status::Ok();
}

// Runs y += alpha * op(A) x.  The stored arrays are read as a CSR matrix `a`
// (for CSC: the CSR of A^T); `transposed` says whether the product needs the
// transpose of those arrays.
Status RunStandardSpmv(asc_sb_context* ctx, const asc_sb_plan* plan,
                       const asc_sb_sparse& m, int op, double alpha, double alpha_imag,
                       const asc_sb_vector& x, const asc_sb_vector& y) {
  const bool csc = m.format == ASC_SB_CSC;
  const bool transposed = (op != ASC_SB_OP_NONE) != csc;
  const ascb_csr a = AsCsr(m, csc);
  const int dtype = Dtype(m.element_kind);
  const ascb_vec xv = AsVec(x), yv = AsVec(y);
  if (!RealKind(m.element_kind)) {
    const bool planned = transposed && plan != nullptr && plan->t_ptr != nullptr;
    const bool exact = ctx->determinism == ASC_SB_DETERMINISTIC;
    ascb_csr rows_of_op = planned ? TransposedCsr(*plan) : a;
    const bool built = transposed && !planned && exact;
    if (built) {
      Status s = TransposedInScratch(ctx, a, ascb::host::ElementBytes(m.element_kind), &rows_of_op);
      if (!s.ok()) return s;
    }
    const int mode = transposed && !planned && !built ? 2 : (exact ? 1 : 0);
    return Launched(ctx,
                    ascb_complex_spmv(ctx->stream, dtype, mode,
                                      op == ASC_SB_OP_CONJUGATE_TRANSPOSE ? 1 : 0, &rows_of_op,
                                      alpha, alpha_imag, &xv, &yv, ctx->sm_count),
                    "CUDA could not launch the complex SpMV kernel");
  }
  if (!transposed) {
    const Choice choice = plan != nullptr ? Choose(ctx, m, plan->variant, plan->lanes)
                                          : ChooseWithoutPlan(ctx, m);
    return RunCsr(ctx, choice, ASCB_STANDARD, a, dtype, alpha, 0.0, xv, yv, nullptr,
                  plan != nullptr ? &plan->part : nullptr);
  }
  if (plan != nullptr && plan->t_ptr != nullptr) {
    const ascb_csr t = TransposedCsr(*plan);
    const Choice choice = Choose(ctx, m);
    return RunCsr(ctx, choice, ASCB_STANDARD, t, dtype, alpha, 0.0, xv, yv, nullptr,
                  &plan->t_part);
  }
  if (ctx->determinism == ASC_SB_DETERMINISTIC) {
    // the reference's order without a plan: the transposed structure in the
    // context's scratch, rebuilt for this call
    ascb_csr t{};
    Status s = TransposedInScratch(ctx, a, ascb::host::ElementBytes(m.element_kind), &t);
    if (!s.ok()) return s;
    return RunCsr(ctx, Choose(ctx, m), ASCB_STANDARD, t, dtype, alpha, 0.0, xv, yv, nullptr,
                  nullptr);
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
  s = ValidateStandardSpmv(ctx, op, m, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (AlphaIsZero(m->element_kind, alpha_real, alpha_imag) || y->extent == 0) {
    return Finish(ctx, Status::Ok());
  }
  return Finish(ctx, RunStandardSpmv(ctx, nullptr, *m, op, alpha_real, alpha_imag, *x, *y));
}

// ---------------------------------------------------------------------------
namespace {

// The row-group kernel's operand rules: row-major B and C whose rows are
// whole 16-byte chunks on 16-byte boundaries.
bool GroupsApply(const asc_sb_dense& b, const asc_sb_dense& c, int kind) {
  const std::int64_t n = kind == ASC_SB_DOUBLE ? 2 : 4;
  return (kind == ASC_SB_FLOAT || kind == ASC_SB_DOUBLE) && b.layout == ASC_SB_ROW_MAJOR &&
         c.layout == ASC_SB_ROW_MAJOR && c.columns % n == 0 && b.leading_dimension % n == 0 &&
         c.leading_dimension % n == 0 &&
         ((reinterpret_cast<std::uintptr_t>(b.data) | reinterpret_cast<std::uintptr_t>(c.data)) &
          15u) == 0;
}

// The staged kernel's operand rules (those of the row groups) and the room
// it needs: two stages of the level's largest stage for this k in one CTA's
// shared memory.  Of the levels that fit, the one that keeps the most CTAs
// per SM, the widest groups (fewest bulk copies) among equals: on a 27-point
// 128^3 stencil (FP32, B200) wide groups of 64 rows take k = 8 from 0.54 to
// 0.28 ms, but at k = 32 their 87 KB stages leave one CTA per SM (0.76 ms
// against 0.61 for the 16-row groups' two).  *level: the tables to run;
// *slots, *entries: the stage's caps.
bool StagedApply(const asc_sb_plan& plan, const asc_sb_dense& b, const asc_sb_dense& c, int kind,
                 int device, const ascb_staged_spmm** level, std::int64_t* slots,
                 std::int64_t* entries) {
  if (!plan.has_staged || !GroupsApply(b, c, kind)) return false;
  const int dtype = Dtype(kind);
  // at most 128 chunks of 16 bytes per row (32 lanes x 4 chunks)
  if (c.columns * static_cast<std::int64_t>(ascb::host::ElementBytes(kind)) > 128 * 16) {
    return false;
  }
  int optin = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) !=
          cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  std::int64_t best_ctas = 0;
  for (int v = ASCB_STAGED_LEVELS - 1; v >= 0; --v) {
    if (!plan.level_ok[v]) continue;
    const ascb_staged_spmm& t = plan.staged[v];
    const std::int64_t* caps = plan.staged_caps[v];
    const int ng = ascb_staged_groups_per_stage(dtype, c.columns, t.group_rows);
    int w = 0;
    while ((1 << w) < ng) ++w;
    const std::size_t stage =
        ascb_staged_stage_bytes(dtype, c.columns, caps[2 * w], caps[2 * w + 1], ng, t.group_rows);
    if (2 * stage > static_cast<std::size_t>(optin)) continue;
    // CTAs per SM by shared memory (1 KB reserved per CTA)
    const std::int64_t ctas =
        std::max<std::int64_t>(1, per_sm / static_cast<std::int64_t>(2 * stage + 1024));
    if (ctas <= best_ctas) continue;
    best_ctas = ctas;
    *level = &t;
    *slots = caps[2 * w];
    *entries = caps[2 * w + 1];
  }
  return best_ctas > 0;
}

// C += alpha * op(A) * B, validated in full before anything is enqueued.  With
// a plan that holds the transposed structure, a transposed product runs the
// stored-order kernel on that structure (bit-exact); without one it scatters.
Status StandardSpmm(asc_sb_context* ctx, const asc_sb_plan* plan, int op, double alpha_real,
                    double alpha_imag, const asc_sb_sparse* m, const asc_sb_dense* b,
                    const asc_sb_dense* c) {
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid");
  }
  if (m == nullptr || b == nullptr || c == nullptr) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA SpMM descriptors cannot be null");
  }
  SparseBytes mb;
  Status s = ascb::host::ValidateSparse(*m, ctx->device, &mb);
  if (!s.ok()) return s;
  Span bs, cs;
  s = ascb::host::ValidateDense(*b, m->element_kind, false, ctx->device, &bs);
  if (!s.ok()) return s;
  s = ascb::host::ValidateDense(*c, m->element_kind, true, ctx->device, &cs);
  if (!s.ok()) return s;
  const std::int64_t inner = op == ASC_SB_OP_NONE ? m->columns : m->rows;
  const std::int64_t rows = op == ASC_SB_OP_NONE ? m->rows : m->columns;
  if (b->rows != inner || c->rows != rows || b->columns != c->columns) {
    return Fail(ASC_SB_SHAPE, "CUDA standardized SpMM matrix extents do not match");
  }
  if (ascb::host::Overlap(bs, cs) || ascb::host::Overlap({m->structure_first, mb.first}, cs) ||
      ascb::host::Overlap({m->structure_second, mb.second}, cs) ||
      ascb::host::Overlap({m->values, mb.values}, cs)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA standardized SpMM output overlaps an input");
  }
  if (AlphaIsZero(m->element_kind, alpha_real, alpha_imag) || c->rows == 0 || c->columns == 0) {
    return Status::Ok();
  }
  const bool csc = m->format == ASC_SB_CSC;
  const bool transposed = (op != ASC_SB_OP_NONE) != csc;
  bool planned = transposed && plan != nullptr && plan->t_ptr != nullptr;
  ascb_csr a = planned ? TransposedCsr(*plan) : AsCsr(*m, csc);
  if (transposed && !planned && ctx->determinism == ASC_SB_DETERMINISTIC) {
    // the reference's order without a plan: the transposed structure in the
    // context's scratch, rebuilt for this call
    ascb_csr t{};
    s = TransposedInScratch(ctx, a, ascb::host::ElementBytes(m->element_kind), &t);
    if (!s.ok()) return s;
    a = t;
    planned = true;
  }
  if (!transposed && !csc && plan != nullptr && plan->block16 &&
      m->element_kind == ASC_SB_FLOAT && ctx->determinism != ASC_SB_DETERMINISTIC &&
      ctx->variant == ASC_SB_VARIANT_AUTO && b->layout == ASC_SB_ROW_MAJOR &&
      c->layout == ASC_SB_ROW_MAJOR) {
    // dense 16 x 16 blocks: tensor cores (3xTF32), within the bound stated in
    // spmm_block16_tc.cu; faster than the CUDA-core kernels at every k
    // measured on B200 (65,536-row 2% block-sparse matrix, k = 8 / 32 / 128:
    // 0.48 / 0.51 / 0.62 ms against 0.80 / 1.05 / 2.04 ms).  The B^T tile
    // images of the call's pre-pass live in the context's scratch.
    unsigned char* tiles = nullptr;
    s = SolveScratch(ctx, RoundUp(ascb_block16_tiles_bytes(a.cols, c->columns), 256), &tiles);
    if (!s.ok()) return s;
    return Launched(ctx,
                    ascb_spmm_block16_tc(ctx->stream, &a, c->columns,
                                         static_cast<const float*>(b->data), b->leading_dimension,
                                         static_cast<float*>(const_cast<void*>(c->data)),
                                         c->leading_dimension, static_cast<float>(alpha_real),
                                         reinterpret_cast<float*>(tiles), ctx->status,
                                         ctx->sm_count),
                    "CUDA could not launch the tensor-core SpMM kernel", 2);
  }
  if (!RealKind(m->element_kind)) {
    const int mode = transposed && !planned ? 2 : (ctx->determinism == ASC_SB_DETERMINISTIC ? 1 : 0);
    return Launched(ctx,
                    ascb_complex_spmm(ctx->stream, Dtype(m->element_kind), mode,
                                      op == ASC_SB_OP_CONJUGATE_TRANSPOSE ? 1 : 0, &a, c->columns,
                                      b->data, b->layout, b->leading_dimension,
                                      const_cast<void*>(c->data), c->layout,
                                      c->leading_dimension, alpha_real, alpha_imag,
                                      ctx->sm_count),
                    "CUDA could not launch the complex SpMM kernel");
  }
  // the staged kernel by default for k >= 8 elements where its stages fit
  // (27-point 128^3 stencil, FP32, B200, contracted / bit-exact: k = 8 0.25 /
  // 0.26 ms against 0.31 / 0.30 row by row, k = 32 0.49 / 0.53 against 0.62 /
  // 0.86, k = 128 2.09 / 2.25 against 2.32 / 2.50); for any k once the
  // autotuner picked it
  std::int64_t st_slots = 0, st_entries = 0;
  const ascb_staged_spmm* st_level = nullptr;
  const bool staged_k = c->columns >= 8;
  if (!transposed && !csc && plan != nullptr && plan->use_staged &&
      (plan->staged_tuned || staged_k) &&
      StagedApply(*plan, *b, *c, m->element_kind, ctx->device, &st_level, &st_slots,
                  &st_entries)) {
    return Launched(ctx,
                    ascb_spmm_staged(ctx->stream, Dtype(m->element_kind),
                                     ctx->determinism == ASC_SB_DETERMINISTIC ? 1 : 0, &a,
                                     st_level, c->columns, b->data, b->leading_dimension,
                                     const_cast<void*>(c->data), c->leading_dimension,
                                     alpha_real, st_slots, st_entries, ctx->status,
                                     ctx->sm_count),
                    "CUDA could not launch the staged SpMM kernel");
  }
  if (!transposed && !csc && plan != nullptr && plan->use_groups &&
      GroupsApply(*b, *c, m->element_kind)) {
    return Launched(ctx,
                    ascb_spmm_groups(ctx->stream, Dtype(m->element_kind),
                                     ctx->determinism == ASC_SB_DETERMINISTIC ? 1 : 0, &a,
                                     &plan->groups, c->columns, b->data, b->leading_dimension,
                                     const_cast<void*>(c->data), c->leading_dimension,
                                     alpha_real, ctx->sm_count),
                    "CUDA could not launch the row-group SpMM kernel");
  }
  return Launched(ctx,
                  ascb_spmm(ctx->stream, Dtype(m->element_kind), transposed && !planned ? 1 : 0,
                            ctx->determinism == ASC_SB_DETERMINISTIC ? 1 : 0, &a, c->columns, b->data, b->layout, b->leading_dimension,
                            const_cast<void*>(c->data), c->layout, c->leading_dimension,
                            alpha_real, ctx->sm_count),
                  "CUDA could not launch the SpMM kernel");
}

}  // namespace

int asc_sb_standard_spmm(asc_sb_context* ctx, int32_t op, double alpha_real, double alpha_imag,
                         const asc_sb_sparse* m, const asc_sb_dense* b, const asc_sb_dense* c) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  return Finish(ctx, StandardSpmm(ctx, nullptr, op, alpha_real, alpha_imag, m, b, c));
}

// ---------------------------------------------------------------------------
int asc_sb_plan_workspace_size(asc_sb_context* ctx, const asc_sb_sparse* m, int32_t flags,
                               size_t* bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (m == nullptr || bytes == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "plan arguments cannot be null"));
  }
  if ((flags & ~(ASC_SB_PLAN_TRANSPOSE | ASC_SB_PLAN_TRIANGULAR | ASC_SB_PLAN_ROW_GROUPS)) != 0) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "unknown plan flags"));
  }
  if (m->rows < 0 || m->columns < 0 || m->nonzeros < 0) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "plan matrix extents cannot be negative"));
  }
  *bytes = PlanLayoutFor(*m, flags).total;
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
  auto* ws = static_cast<unsigned char*>(workspace);
  s = BuildPartitions(ctx, a, ws, &plan->part);
  if (s.ok() && (flags & ASC_SB_PLAN_TRANSPOSE)) {
    const PlanLayout l = PlanLayoutFor(*m, flags);
    plan->t_ptr = reinterpret_cast<std::int64_t*>(ws + l.t_ptr);
    plan->t_idx = reinterpret_cast<std::int64_t*>(ws + l.t_idx);
    plan->t_perm = reinterpret_cast<std::int64_t*>(ws + l.t_perm);
    plan->t_val = ws + l.t_val;
    s = BuildTransposed(ctx, a, ascb::host::ElementBytes(m->element_kind), plan->t_ptr,
                        plan->t_idx, plan->t_perm, plan->t_val, ws + l.sort,
                        reinterpret_cast<std::int64_t*>(ws + l.outer_of));
    if (s.ok()) s = BuildPartitions(ctx, TransposedCsr(*plan), ws + l.t_part, &plan->t_part);
  }
  if (flags & ASC_SB_PLAN_TRIANGULAR) {
    plan->solve = ws + PlanLayoutFor(*m, flags).solve;
    plan->analysis = ws + PlanLayoutFor(*m, flags).analysis;
  }
  if (s.ok() && m->format == ASC_SB_CSR && m->element_kind == ASC_SB_FLOAT && m->rows > 0 &&
      m->rows % 16 == 0 && m->nonzeros > 0 &&
      (reinterpret_cast<std::uintptr_t>(m->values) & 15u) == 0) {
    s = DetectBlocks(ctx, a, reinterpret_cast<int*>(ws + PlanLayoutFor(*m, flags).flag), plan);
  }
  // (run offsets are 32-bit: groups are built below 2^32 stored entries)
  if (s.ok() && (flags & ASC_SB_PLAN_ROW_GROUPS) && m->format == ASC_SB_CSR &&
      RealKind(m->element_kind) && m->rows > 0 && m->nonzeros < (std::int64_t{1} << 32)) {
    plan->groups_mem = ws + PlanLayoutFor(*m, flags).groups;
    plan->staged_mem = ws + PlanLayoutFor(*m, flags).staged;
    s = BuildRowGroups(ctx, plan, 16);
    if (s.ok()) s = BuildStaged(ctx, plan);
    if (s.ok() && kDefaultRowsPerGroup != 16) s = BuildRowGroups(ctx, plan, kDefaultRowsPerGroup);
    // row groups only where the autotuner measured them faster: on B200 they
    // lose to the row-by-row kernel on stencils (27-point 128^3, k = 32:
    // 2.2 ms with R = 8 against 0.62 ms) and win on dense-block rows in
    // DETERMINISTIC mode (16 x 16 blocks, k = 32: 0.93 ms with R = 16
    // against 1.29 ms)
    plan->use_groups = false;
  }
  if (s.ok() && ctx->selector != nullptr && ctx->determinism != ASC_SB_DETERMINISTIC &&
      ctx->variant == ASC_SB_VARIANT_AUTO && RealKind(m->element_kind)) {
    s = SelectVariant(ctx, plan);
  }
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
  if (plan->t_ptr == nullptr) return Finish(ctx, Status::Ok());
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  // the transposed values are a gather of the stored ones through t_perm
  return Finish(ctx, Launched(ctx,
                              ascb_permute_entries(
                                  ctx->stream, plan->t_perm, plan->matrix.nonzeros, nullptr, 0,
                                  nullptr, plan->matrix.values, plan->t_val,
                                  static_cast<int>(ascb::host::ElementBytes(plan->matrix.element_kind)),
                                  ctx->sm_count),
                              "CUDA could not launch the entry permutation kernel"));
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
  const Choice choice = Choose(ctx, plan->matrix, plan->variant, plan->lanes);
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
  s = ValidateStandardSpmv(ctx, op, &plan->matrix, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (AlphaIsZero(plan->matrix.element_kind, alpha_real, alpha_imag) || y->extent == 0) {
    return Finish(ctx, Status::Ok());
  }
  return Finish(ctx,
                RunStandardSpmv(ctx, plan, plan->matrix, op, alpha_real, alpha_imag, *x, *y));
}

int asc_sb_plan_standard_spmm(asc_sb_context* ctx, const asc_sb_plan* plan, int32_t op,
                              double alpha_real, double alpha_imag, const asc_sb_dense* b,
                              const asc_sb_dense* c) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  return Finish(ctx, StandardSpmm(ctx, plan, op, alpha_real, alpha_imag, &plan->matrix, b, c));
}

// ---------------------------------------------------------------------------
// Format conversion on the device.

namespace {

struct ConvertLayout {
  std::size_t perm = 0, outer_of = 0, sort = 0, total = 0;
};

ConvertLayout ConvertLayoutFor(std::int64_t nnz, std::int64_t destination_outer) {
  ConvertLayout l;
  std::size_t at = 0;
  l.perm = at;
  at += EntryBytes(nnz, 8);
  l.outer_of = at;
  at += EntryBytes(nnz, 8);
  l.sort = at;
  at += RoundUp(ascb_sort_workspace_bytes(nnz, destination_outer), 256);
  l.total = at;
  return l;
}

// The destination of a conversion: caller-allocated device arrays of the
// other format, validated like any sparse operand (it is canonical once
// written), disjoint from the source and the workspace.
Status ValidateDestination(asc_sb_context* ctx, const asc_sb_sparse* d, int element_kind,
                           std::int64_t rows, std::int64_t columns, std::int64_t nnz,
                           SparseBytes* bytes) {
  if (d == nullptr) return Fail(ASC_SB_INVALID_ARGUMENT, "conversion destination cannot be null");
  if (d->element_kind != element_kind) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "conversion source and destination elements must match");
  }
  if (d->rows != rows || d->columns != columns || d->nonzeros != nnz) {
    return Fail(ASC_SB_SHAPE, "conversion destination shape does not match the source");
  }
  asc_sb_sparse trusted = *d;
  trusted.canonical_structure_trusted = 1;
  return ascb::host::ValidateSparse(trusted, ctx->device, bytes);
}

Status ValidateConvertWorkspace(asc_sb_context* ctx, void* workspace, std::size_t bytes,
                                std::size_t need) {
  if (bytes < need || (need != 0 && workspace == nullptr)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "conversion workspace is missing or too small");
  }
  if ((reinterpret_cast<std::uintptr_t>(workspace) & 255u) != 0) {
    return Fail(ASC_SB_MEMORY_ACCESS, "conversion workspace must be 256-byte aligned");
  }
  return ascb::host::ValidateDevicePointer(workspace, bytes, ctx->device,
                                           "CUDA could not inspect conversion workspace");
}

bool DestinationOverlaps(const asc_sb_sparse& d, const SparseBytes& db, Span other) {
  return ascb::host::Overlap({d.structure_first, db.first}, other) ||
         ascb::host::Overlap({d.structure_second, db.second}, other) ||
         ascb::host::Overlap({d.values, db.values}, other);
}

}  // namespace

int asc_sb_convert_workspace_size(asc_sb_context* ctx, int64_t rows, int64_t columns,
                                  int64_t nonzeros, int32_t destination_format, size_t* bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (bytes == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "bytes cannot be null"));
  if (destination_format != ASC_SB_CSR && destination_format != ASC_SB_CSC) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "conversions produce CSR or CSC"));
  }
  if (rows < 0 || columns < 0 || nonzeros < 0) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "conversion extents cannot be negative"));
  }
  *bytes = ConvertLayoutFor(nonzeros, destination_format == ASC_SB_CSR ? rows : columns).total;
  return Finish(ctx, Status::Ok());
}

int asc_sb_convert_compressed(asc_sb_context* ctx, const asc_sb_sparse* source,
                              const asc_sb_sparse* destination, void* workspace,
                              size_t workspace_bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (source == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "conversion source cannot be null"));
  }
  SparseBytes sb, db;
  s = ascb::host::ValidateSparse(*source, ctx->device, &sb);
  if (!s.ok()) return Finish(ctx, s);
  s = ValidateDestination(ctx, destination, source->element_kind, source->rows, source->columns,
                          source->nonzeros, &db);
  if (!s.ok()) return Finish(ctx, s);
  if (destination->format == source->format) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                            "a compressed conversion goes from CSR to CSC or from CSC to CSR"));
  }
  const std::int64_t dest_outer =
      destination->format == ASC_SB_CSR ? source->rows : source->columns;
  const ConvertLayout l = ConvertLayoutFor(source->nonzeros, dest_outer);
  s = ValidateConvertWorkspace(ctx, workspace, workspace_bytes, l.total);
  if (!s.ok()) return Finish(ctx, s);
  const Span ws{workspace, workspace_bytes};
  if (DestinationOverlaps(*destination, db, {source->structure_first, sb.first}) ||
      DestinationOverlaps(*destination, db, {source->structure_second, sb.second}) ||
      DestinationOverlaps(*destination, db, {source->values, sb.values}) ||
      DestinationOverlaps(*destination, db, ws) ||
      ascb::host::Overlap({source->structure_first, sb.first}, ws) ||
      ascb::host::Overlap({source->structure_second, sb.second}, ws) ||
      ascb::host::Overlap({source->values, sb.values}, ws)) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                            "conversion destination and workspace must not overlap any operand"));
  }
  // the source read as CSR arrays: outer = its outer extent, keys = its inner
  // indices, which become the destination's outer indices
  const ascb_csr a = AsCsr(*source, source->format == ASC_SB_CSC);
  auto* w = static_cast<unsigned char*>(workspace);
  auto* perm = reinterpret_cast<std::int64_t*>(w + l.perm);
  s = BuildTransposed(ctx, a, ascb::host::ElementBytes(source->element_kind),
                      static_cast<std::int64_t*>(const_cast<void*>(destination->structure_first)),
                      static_cast<std::int64_t*>(const_cast<void*>(destination->structure_second)),
                      perm, const_cast<void*>(destination->values), w + l.sort,
                      reinterpret_cast<std::int64_t*>(w + l.outer_of));
  return Finish(ctx, s);
}

int asc_sb_convert_coordinates(asc_sb_context* ctx, const int64_t* coordinates,
                               const void* values, int32_t element_kind, int64_t rows,
                               int64_t columns, int64_t nonzeros,
                               const asc_sb_sparse* destination, void* workspace,
                               size_t workspace_bytes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (rows < 0 || columns < 0 || nonzeros < 0) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "conversion extents cannot be negative"));
  }
  SparseBytes db;
  s = ValidateDestination(ctx, destination, element_kind, rows, columns, nonzeros, &db);
  if (!s.ok()) return Finish(ctx, s);
  const std::size_t element = ascb::host::ElementBytes(element_kind);
  const Span cs{coordinates, static_cast<std::size_t>(nonzeros) * 16};
  const Span vs{values, static_cast<std::size_t>(nonzeros) * element};
  if (nonzeros > 0) {
    s = ascb::host::ValidateAddress(coordinates, cs.bytes, 8, "coordinate storage is incomplete",
                                    "coordinate storage is misaligned");
    if (!s.ok()) return Finish(ctx, s);
    s = ascb::host::ValidateAddress(values, vs.bytes, element > 8 ? 8 : element,
                                    "coordinate value storage is incomplete",
                                    "coordinate value storage is misaligned");
    if (!s.ok()) return Finish(ctx, s);
    s = ascb::host::ValidateDevicePointer(coordinates, cs.bytes, ctx->device,
                                          "CUDA could not inspect coordinate storage");
    if (!s.ok()) return Finish(ctx, s);
    s = ascb::host::ValidateDevicePointer(values, vs.bytes, ctx->device,
                                          "CUDA could not inspect coordinate value storage");
    if (!s.ok()) return Finish(ctx, s);
  }
  const bool to_csr = destination->format == ASC_SB_CSR;
  const ConvertLayout l = ConvertLayoutFor(nonzeros, to_csr ? rows : columns);
  s = ValidateConvertWorkspace(ctx, workspace, workspace_bytes, l.total);
  if (!s.ok()) return Finish(ctx, s);
  const Span ws{workspace, workspace_bytes};
  if (DestinationOverlaps(*destination, db, cs) || DestinationOverlaps(*destination, db, vs) ||
      DestinationOverlaps(*destination, db, ws) || ascb::host::Overlap(cs, ws) ||
      ascb::host::Overlap(vs, ws)) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                            "conversion destination and workspace must not overlap any operand"));
  }
  auto* w = static_cast<unsigned char*>(workspace);
  auto* perm = reinterpret_cast<std::int64_t*>(w + l.perm);
  auto* offsets = static_cast<std::int64_t*>(const_cast<void*>(destination->structure_first));
  // coordinates are (row, column) pairs: the destination's outer index is the
  // row for CSR and the column for CSC, the other one becomes the inner index
  s = Launched(ctx,
               ascb_stable_sort(ctx->stream, coordinates + (to_csr ? 0 : 1), 2, nonzeros,
                                to_csr ? rows : columns, offsets, perm, w + l.sort),
               "CUDA could not launch the conversion sort");
  if (!s.ok()) return Finish(ctx, s);
  s = Launched(ctx,
               ascb_permute_entries(
                   ctx->stream, perm, nonzeros, coordinates + (to_csr ? 1 : 0), 2,
                   static_cast<std::int64_t*>(const_cast<void*>(destination->structure_second)),
                   values, const_cast<void*>(destination->values), static_cast<int>(element),
                   ctx->sm_count),
               "CUDA could not launch the entry permutation kernel");
  return Finish(ctx, s);
}

// ---------------------------------------------------------------------------
// Level-1 on an indexed vector.

int asc_sb_standard_level1(asc_sb_context* ctx, int32_t operation, int32_t conjugation,
                           double alpha_real, double alpha_imag,
                           const asc_sb_indexed_vector* sparse, const asc_sb_vector* dense,
                           const asc_sb_vector* result) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (conjugation != ASC_SB_UNCONJUGATED && conjugation != ASC_SB_CONJUGATED) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS conjugation is invalid"));
  }
  if (operation < ASC_SB_L1_DOT || operation > ASC_SB_L1_SCATTER) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS level-one operation is invalid"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (sparse == nullptr || dense == nullptr ||
      (operation == ASC_SB_L1_DOT && result == nullptr)) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "level-one descriptors cannot be null"));
  }
  // ValidateIndexedDevice (operations.cc:278-332 style rules)
  const bool sparse_writable =
      operation == ASC_SB_L1_GATHER || operation == ASC_SB_L1_GATHER_ZERO;
  if (sparse->memory_space != ASC_SB_DEVICE) {
    return Finish(ctx, Fail(ASC_SB_MEMORY_ACCESS, "Sparse CUDA indexed vectors require device storage"));
  }
  if (sparse->element_kind < ASC_SB_FLOAT || sparse->element_kind > ASC_SB_COMPLEX_DOUBLE) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA scalar kind is invalid"));
  }
  if (!sparse->canonical_structure_trusted) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                            "Sparse CUDA indexed vectors require trusted canonical structure"));
  }
  if (sparse_writable && !sparse->writable) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse CUDA indexed vector is not writable"));
  }
  if (sparse->nonzeros < 0 || sparse->dense_extent < 0 ||
      sparse->nonzeros > sparse->dense_extent) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "Sparse CUDA indexed vector extents are invalid"));
  }
  const std::size_t element = ascb::host::ElementBytes(sparse->element_kind);
  const Span idx_span{sparse->indices, static_cast<std::size_t>(sparse->nonzeros) * 8};
  const Span val_span{sparse->values, static_cast<std::size_t>(sparse->nonzeros) * element};
  if (sparse->nonzeros > 0) {
    s = ascb::host::ValidateAddress(sparse->indices, idx_span.bytes, 8,
                                    "Sparse CUDA index storage is incomplete",
                                    "Sparse CUDA index storage is misaligned");
    if (s.ok()) {
      s = ascb::host::ValidateAddress(sparse->values, val_span.bytes, element > 8 ? 8 : element,
                                      "Sparse CUDA value storage is incomplete",
                                      "Sparse CUDA value storage is misaligned");
    }
    if (s.ok()) {
      s = ascb::host::ValidateDevicePointer(sparse->indices, idx_span.bytes, ctx->device,
                                            "CUDA could not inspect sparse operand storage");
    }
    if (s.ok()) {
      s = ascb::host::ValidateDevicePointer(sparse->values, val_span.bytes, ctx->device,
                                            "CUDA could not inspect sparse operand storage");
    }
    if (!s.ok()) return Finish(ctx, s);
    if (ascb::host::Overlap(idx_span, val_span)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                              "Sparse CUDA descriptor storage spans cannot overlap"));
    }
  }
  const bool dense_writable = operation == ASC_SB_L1_AXPY ||
                              operation == ASC_SB_L1_GATHER_ZERO ||
                              operation == ASC_SB_L1_SCATTER;
  Span ds;
  s = ascb::host::ValidateVector(*dense, sparse->element_kind, dense_writable, ctx->device, &ds);
  if (!s.ok()) return Finish(ctx, s);
  if (dense->extent != sparse->dense_extent) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "CUDA Sparse BLAS level-one vector extents do not match"));
  }
  if (operation != ASC_SB_L1_DOT &&
      (ascb::host::Overlap(val_span, ds) || ascb::host::Overlap(idx_span, ds))) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT,
                            "CUDA Sparse BLAS level-one writable operands overlap"));
  }
  Span rs;
  if (operation == ASC_SB_L1_DOT) {
    s = ascb::host::ValidateVector(*result, sparse->element_kind, true, ctx->device, &rs);
    if (!s.ok()) return Finish(ctx, s);
    if (result->extent != 1) {
      return Finish(ctx, Fail(ASC_SB_SHAPE, "CUDA sparse dot requires one result element"));
    }
    if (ascb::host::Overlap(rs, ds) || ascb::host::Overlap(rs, idx_span) ||
        ascb::host::Overlap(rs, val_span)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "CUDA sparse dot result overlaps an input"));
    }
  }
  if (operation == ASC_SB_L1_AXPY &&
      AlphaIsZero(sparse->element_kind, alpha_real, alpha_imag)) {
    return Finish(ctx, Status::Ok());
  }
  if (operation != ASC_SB_L1_DOT && sparse->nonzeros == 0) return Finish(ctx, Status::Ok());
  return Finish(ctx, Launched(ctx,
                              ascb_level1(ctx->stream, Dtype(sparse->element_kind), operation,
                                          conjugation, ctx->determinism == ASC_SB_DETERMINISTIC,
                                          static_cast<const std::int64_t*>(sparse->indices),
                                          const_cast<void*>(sparse->values), sparse->nonzeros,
                                          const_cast<void*>(dense->data), dense->stride,
                                          result != nullptr ? const_cast<void*>(result->data)
                                                            : nullptr,
                                          alpha_real, alpha_imag, ctx->scratch, ctx->sm_count),
                              "CUDA could not launch the level-one kernel"));
}

// ---------------------------------------------------------------------------
// Sparse triangular solve.

namespace {

// Grows the context's solve buffer to `bytes`.  A larger buffer replaces the
// old one only after the stream has finished with it.
Status SolveScratch(asc_sb_context* ctx, std::size_t bytes, unsigned char** out) {
  if (ctx->solve_mem.bytes < bytes) {
    if (ctx->solve_mem.ptr != nullptr) {
      if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        (void)cudaGetLastError();
        return Fail(ASC_SB_PROVIDER, "CUDA could not drain the stream before growing scratch");
      }
      ascb::host::Release(&ctx->solve_mem);
    }
    if (!ascb::host::Acquire(ctx->allocator, bytes, ASC_SB_DEVICE, &ctx->solve_mem)) {
      return Fail(ASC_SB_ALLOCATION, "could not allocate triangular-solve scratch");
    }
  }
  *out = static_cast<unsigned char*>(ctx->solve_mem.ptr);
  return Status::Ok();
}

// StandardTriangularSolveErased (operations.cc:1380-1451): validation in the
// facet's order, then one sync-free solve on the CSR arrays of op(A).
Status TriangularSolve(asc_sb_context* ctx, const asc_sb_plan* plan, int op, double alpha_real,
                       double alpha_imag, const asc_sb_sparse* m, int triangle, int diagonal,
                       const asc_sb_dense* rhs) {
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid");
  }
  if (triangle != ASC_SB_UPPER && triangle != ASC_SB_LOWER) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "A sparse BLAS triangle value is invalid");
  }
  if (diagonal != ASC_SB_NON_UNIT && diagonal != ASC_SB_UNIT) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "A sparse BLAS diagonal value is invalid");
  }
  if (m == nullptr || rhs == nullptr) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA triangular-solve descriptors cannot be null");
  }
  if (m->format != ASC_SB_CSR || m->rows != m->columns) {
    return Fail(ASC_SB_SHAPE, "CUDA triangular solve requires square CSR storage");
  }
  SparseBytes mb;
  Status s = ascb::host::ValidateSparse(*m, ctx->device, &mb);
  if (!s.ok()) return s;
  Span rs;
  s = ascb::host::ValidateDense(*rhs, m->element_kind, true, ctx->device, &rs);
  if (!s.ok()) return s;
  if (rhs->rows != m->rows) {
    return Fail(ASC_SB_SHAPE, "CUDA triangular right-hand-side extent does not match");
  }
  if (ascb::host::Overlap({m->structure_first, mb.first}, rs) ||
      ascb::host::Overlap({m->structure_second, mb.second}, rs) ||
      ascb::host::Overlap({m->values, mb.values}, rs)) {
    return Fail(ASC_SB_INVALID_ARGUMENT, "CUDA triangular right-hand sides overlap the matrix");
  }
  const std::int64_t n = m->rows;
  const bool transposed = op != ASC_SB_OP_NONE;
  if (plan != nullptr) {
    if (plan->solve == nullptr) {
      return Fail(ASC_SB_INVALID_STATE, "the plan holds no triangular-solve state");
    }
    if (transposed && plan->t_ptr == nullptr) {
      return Fail(ASC_SB_INVALID_STATE, "a transposed solve needs a plan with the transposed structure");
    }
  }
  if (n == 0 || rhs->columns == 0) return Status::Ok();
  const bool alpha_zero = AlphaIsZero(m->element_kind, alpha_real, alpha_imag);
  ascb_csr op_csr = AsCsr(*m, false);
  unsigned char* control = nullptr;
  if (plan != nullptr) {
    control = plan->solve;
    if (transposed) op_csr = TransposedCsr(*plan);
  } else {
    const std::size_t element = ascb::host::ElementBytes(m->element_kind);
    const std::size_t flags =
        RoundUp(ascb_trsv_scratch_bytes(n, static_cast<int>(element)), 256);
    const std::int64_t nnz = m->nonzeros;
    std::size_t total = flags;
    std::size_t t_ptr = 0, t_idx = 0, t_perm = 0, t_val = 0, sort = 0, outer_of = 0;
    if (transposed && !alpha_zero) {
      t_ptr = total;
      total += RoundUp(static_cast<std::size_t>(n + 1) * 8, 256);
      t_idx = total;
      total += EntryBytes(nnz, 8);
      t_perm = total;
      total += EntryBytes(nnz, 8);
      t_val = total;
      total += EntryBytes(nnz, element);
      sort = total;
      total += RoundUp(ascb_sort_workspace_bytes(nnz, n), 256);
      outer_of = total;
      total += EntryBytes(nnz, 8);
    }
    s = SolveScratch(ctx, total, &control);
    if (!s.ok()) return s;
    if (transposed && !alpha_zero) {
      auto* tp = reinterpret_cast<std::int64_t*>(control + t_ptr);
      auto* ti = reinterpret_cast<std::int64_t*>(control + t_idx);
      s = BuildTransposed(ctx, op_csr, element, tp, ti,
                          reinterpret_cast<std::int64_t*>(control + t_perm), control + t_val,
                          control + sort, reinterpret_cast<std::int64_t*>(control + outer_of));
      if (!s.ok()) return s;
      op_csr.ptr = tp;
      op_csr.idx = ti;
      op_csr.val = control + t_val;
    }
  }
  ascb_trsv t{};
  t.ptr = op_csr.ptr;
  t.idx = op_csr.idx;
  t.val = op_csr.val;
  t.n = n;
  t.lower = transposed ? triangle == ASC_SB_UPPER : triangle == ASC_SB_LOWER;
  t.unit = diagonal == ASC_SB_UNIT;
  t.conj = op == ASC_SB_OP_CONJUGATE_TRANSPOSE && !RealKind(m->element_kind);
  t.row_major = rhs->layout == ASC_SB_ROW_MAJOR;
  t.x = const_cast<void*>(rhs->data);
  t.ld = rhs->leading_dimension;
  t.k = rhs->columns;
  t.control = control;
  t.pub = control + 16;
  if (plan != nullptr && plan->analysed && plan->analysis_transposed == transposed &&
      plan->analysis_lower == (t.lower != 0)) {
    t.order = plan->order;
    t.position = plan->position;
  }
  t.status = ctx->status;
  t.wait_ns = ctx->wait_ns;
  return Launched(ctx,
                  ascb_sptrsv(ctx->stream, Dtype(m->element_kind),
                              ctx->determinism == ASC_SB_DETERMINISTIC, alpha_zero, &t,
                              alpha_real, alpha_imag, ctx->sm_count),
                  "CUDA could not launch the triangular solve");
}

}  // namespace

int asc_sb_standard_triangular_solve(asc_sb_context* ctx, int32_t op, double alpha_real,
                                     double alpha_imag, const asc_sb_sparse* matrix,
                                     int32_t triangle, int32_t diagonal,
                                     const asc_sb_dense* right_hand_sides) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  return Finish(ctx, TriangularSolve(ctx, nullptr, op, alpha_real, alpha_imag, matrix, triangle,
                                     diagonal, right_hand_sides));
}

int asc_sb_plan_triangular_analysis(asc_sb_context* ctx, asc_sb_plan* plan, int32_t op,
                                    int32_t triangle) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  if (op != ASC_SB_OP_NONE && op != ASC_SB_OP_TRANSPOSE && op != ASC_SB_OP_CONJUGATE_TRANSPOSE) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Sparse BLAS transpose mode is invalid"));
  }
  if (triangle != ASC_SB_UPPER && triangle != ASC_SB_LOWER) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "A sparse BLAS triangle value is invalid"));
  }
  const asc_sb_sparse& m = plan->matrix;
  if (m.format != ASC_SB_CSR || m.rows != m.columns) {
    return Finish(ctx, Fail(ASC_SB_SHAPE, "CUDA triangular solve requires square CSR storage"));
  }
  const bool transposed = op != ASC_SB_OP_NONE;
  if (plan->analysis == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE, "the plan holds no triangular-solve state"));
  }
  if (transposed && plan->t_ptr == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE,
                            "a transposed solve needs a plan with the transposed structure"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  const ascb_csr op_csr = transposed ? TransposedCsr(*plan) : AsCsr(m, false);
  ascb_trsv t{};
  t.ptr = op_csr.ptr;
  t.idx = op_csr.idx;
  t.n = m.rows;
  t.lower = transposed ? triangle == ASC_SB_UPPER : triangle == ASC_SB_LOWER;
  t.control = plan->solve;
  t.status = ctx->status;
  t.wait_ns = ctx->wait_ns;
  std::int64_t* order = nullptr;
  std::int64_t* position = nullptr;
  plan->analysed = false;
  s = Launched(ctx, ascb_trsv_analysis(ctx->stream, &t, plan->analysis, &order, &position,
                                       ctx->sm_count),
               "CUDA could not launch the triangular-solve analysis");
  if (!s.ok()) return Finish(ctx, s);
  plan->order = order;
  plan->position = position;
  plan->analysis_transposed = transposed;
  plan->analysis_lower = t.lower != 0;
  plan->analysed = true;
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_triangular_solve(asc_sb_context* ctx, const asc_sb_plan* plan, int32_t op,
                                 double alpha_real, double alpha_imag, int32_t triangle,
                                 int32_t diagonal, const asc_sb_dense* right_hand_sides) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  return Finish(ctx, TriangularSolve(ctx, plan, op, alpha_real, alpha_imag, &plan->matrix,
                                     triangle, diagonal, right_hand_sides));
}

// ---------------------------------------------------------------------------
// Learned variant selector.

int64_t asc_sb_selector_param_count(int32_t n_variants) {
  return n_variants >= 1 && n_variants <= kSelMaxOutputs ? ascb_mlp_param_count(n_variants) : -1;
}

int asc_sb_context_set_selector(asc_sb_context* ctx, int32_t n_variants, const float* params,
                                const int32_t* variants, const int32_t* lanes) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (params == nullptr) {  // remove
    (void)cudaStreamSynchronize(ctx->stream);
    ascb::host::Release(&ctx->selector_mem);
    ctx->selector = nullptr;
    ctx->selector_outputs = 0;
    ForgetPicks(ctx);
    return Finish(ctx, Status::Ok());
  }
  if (n_variants < 1 || n_variants > kSelMaxOutputs || variants == nullptr || lanes == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "selector arguments are invalid"));
  }
  for (int i = 0; i < n_variants; ++i) {
    if (!ValidVariant(variants[i], variants[i] == ASC_SB_VARIANT_VECTOR ? lanes[i] : 1)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "selector names an unknown variant"));
    }
  }
  const std::size_t count = static_cast<std::size_t>(ascb_mlp_param_count(n_variants));
  const std::size_t bytes = (kSelParams + count) * sizeof(float);
  ascb::host::Block mem;
  if (!ascb::host::Acquire(ctx->allocator, bytes, ASC_SB_DEVICE, &mem)) {
    return Finish(ctx, Fail(ASC_SB_ALLOCATION, "could not allocate the selector's parameters"));
  }
  float* dev = static_cast<float*>(mem.ptr);
  const cudaError_t e = cudaMemcpyAsync(dev + kSelParams, params, count * sizeof(float),
                                        cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    (void)cudaGetLastError();
    ascb::host::Release(&mem);
    return Finish(ctx, Fail(ASC_SB_MEMORY_TRANSFER, "could not copy the selector's parameters"));
  }
  // the new parameters replace the old ones only once they are in place
  ascb::host::Release(&ctx->selector_mem);
  ctx->selector_mem = mem;
  ctx->selector = dev;
  ForgetPicks(ctx);
  ctx->selector_outputs = n_variants;
  ctx->selector_variant.assign(variants, variants + n_variants);
  ctx->selector_lanes.assign(lanes, lanes + n_variants);
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_properties(const asc_sb_plan* plan, int32_t* properties) {
  if (plan == nullptr || properties == nullptr) return ASC_SB_INVALID_ARGUMENT;
  *properties = (plan->t_ptr != nullptr ? ASC_SB_PLAN_HAS_TRANSPOSE : 0) |
                (plan->block16 ? ASC_SB_PLAN_HAS_BLOCKS16 : 0) |
                (plan->use_groups ? ASC_SB_PLAN_HAS_ROW_GROUPS : 0) |
                (plan->use_staged ? ASC_SB_PLAN_HAS_STAGED_SPMM : 0);
  return ASC_SB_OK;
}

int asc_sb_plan_variant(const asc_sb_plan* plan, int32_t* variant, int32_t* lanes) {
  if (plan == nullptr || variant == nullptr || lanes == nullptr) return ASC_SB_INVALID_ARGUMENT;
  *variant = plan->variant >= -1 ? plan->variant : ASC_SB_VARIANT_AUTO;
  *lanes = plan->lanes;
  return ASC_SB_OK;
}

int asc_sb_plan_spmm_autotune(asc_sb_context* ctx, asc_sb_plan* plan, double alpha,
                              const asc_sb_dense* b, const asc_sb_dense* c, int32_t reps,
                              float* best_ms, int32_t* rows_per_group) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr || b == nullptr || c == nullptr || reps < 1 || best_ms == nullptr ||
      rows_per_group == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "SpMM autotune arguments are invalid"));
  }
  if (plan->groups_mem == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE,
                            "SpMM autotuning needs a plan created with ASC_SB_PLAN_ROW_GROUPS"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  // candidates: 0 = the row-by-row kernel, ASC_SB_SPMM_STAGED = the
  // TMA-staged kernel, else R rows per group
  const int candidates[] = {0, ASC_SB_SPMM_STAGED, 2, 4, 8, 16, 32};
  std::int64_t st_slots = 0, st_entries = 0;
  const ascb_staged_spmm* st_level = nullptr;
  const bool staged_ok = StagedApply(*plan, *b, *c, plan->matrix.element_kind, ctx->device,
                                     &st_level, &st_slots, &st_entries);
  plan->tuned_count = 0;
  cudaEvent_t start = nullptr, stop = nullptr;
  cudaError_t e = cudaEventCreate(&start);
  if (e == cudaSuccess) e = cudaEventCreate(&stop);
  int best = 0;
  bool have_best = false;
  float best_time = 0.0f;
  for (int rg : candidates) {
    if (!s.ok() || e != cudaSuccess) break;
    if (rg == ASC_SB_SPMM_STAGED && !staged_ok) continue;
    if (rg > 0 && plan->groups.rows_per_group != rg) s = BuildRowGroups(ctx, plan, rg);
    if (!s.ok()) break;
    plan->use_groups = rg > 0;
    plan->use_staged = rg == ASC_SB_SPMM_STAGED;
    plan->staged_tuned = rg == ASC_SB_SPMM_STAGED;
    s = StandardSpmm(ctx, plan, ASC_SB_OP_NONE, alpha, 0.0, &plan->matrix, b, c);  // warm-up
    if (s.ok()) e = cudaEventRecord(start, ctx->stream);
    for (int r = 0; r < reps && s.ok() && e == cudaSuccess; ++r) {
      s = StandardSpmm(ctx, plan, ASC_SB_OP_NONE, alpha, 0.0, &plan->matrix, b, c);
    }
    if (s.ok() && e == cudaSuccess) e = cudaEventRecord(stop, ctx->stream);
    if (s.ok() && e == cudaSuccess) e = cudaEventSynchronize(stop);
    float t = 0.0f;
    if (s.ok() && e == cudaSuccess) e = cudaEventElapsedTime(&t, start, stop);
    if (s.ok() && e == cudaSuccess && plan->tuned_count < 8) {
      plan->tuned_candidate[plan->tuned_count] = rg;
      plan->tuned_ms[plan->tuned_count] = t / static_cast<float>(reps);
      ++plan->tuned_count;
    }
    if (s.ok() && e == cudaSuccess && (!have_best || t < best_time)) {
      best = rg;
      best_time = t;
      have_best = true;
    }
  }
  if (start != nullptr) (void)cudaEventDestroy(start);
  if (stop != nullptr) (void)cudaEventDestroy(stop);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    s = {ASC_SB_PROVIDER, std::string("CUDA SpMM autotuning failed: ") + cudaGetErrorString(e)};
  }
  if (s.ok() && best > 0 && plan->groups.rows_per_group != best) s = BuildRowGroups(ctx, plan, best);
  if (!s.ok()) return Finish(ctx, s);
  plan->use_groups = best > 0;
  plan->use_staged = best == ASC_SB_SPMM_STAGED;
  plan->staged_tuned = best == ASC_SB_SPMM_STAGED;
  *best_ms = best_time / static_cast<float>(reps);
  *rows_per_group = best;
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_set_spmm(asc_sb_context* ctx, asc_sb_plan* plan, int32_t choice) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "null plan"));
  if (plan->groups_mem == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE,
                            "choosing the SpMM kernel needs a plan created with "
                            "ASC_SB_PLAN_ROW_GROUPS"));
  }
  const bool valid = choice == ASC_SB_SPMM_AUTO || choice == ASC_SB_SPMM_STAGED || choice == 0 ||
                     choice == 2 || choice == 4 || choice == 8 || choice == 16 || choice == 32;
  if (!valid) return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "unknown SpMM kernel choice"));
  if (choice == ASC_SB_SPMM_STAGED && !plan->has_staged) {
    return Finish(ctx, Fail(ASC_SB_INVALID_STATE, "the plan holds no staged SpMM tables"));
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  if (choice > 0 && plan->groups.rows_per_group != choice) {
    s = BuildRowGroups(ctx, plan, choice);
    if (!s.ok()) return Finish(ctx, s);
  }
  plan->use_groups = choice > 0;
  plan->use_staged = choice == ASC_SB_SPMM_STAGED ||
                     (choice == ASC_SB_SPMM_AUTO && plan->has_staged &&
                      4 * plan->matrix.nonzeros >= 5 * plan->staged_slots);
  plan->staged_tuned = choice == ASC_SB_SPMM_STAGED;
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_spmm_stage_rows(asc_sb_context* ctx, const asc_sb_plan* plan, int64_t k,
                                int64_t* rows) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr || rows == nullptr || k < 0) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "stage-rows arguments are invalid"));
  }
  *rows = 0;
  asc_sb_dense b{}, c{};
  b.layout = c.layout = ASC_SB_ROW_MAJOR;
  b.element_kind = c.element_kind = plan->matrix.element_kind;
  b.columns = c.columns = k;
  b.leading_dimension = c.leading_dimension = k;
  const ascb_staged_spmm* level = nullptr;
  std::int64_t slots = 0, entries = 0;
  if (k > 0 && StagedApply(*plan, b, c, plan->matrix.element_kind, ctx->device, &level, &slots,
                           &entries)) {
    *rows = level->group_rows;
  }
  return Finish(ctx, Status::Ok());
}

int asc_sb_plan_spmm_tuning(const asc_sb_plan* plan, int32_t capacity, int32_t* count,
                            int32_t* candidates, float* ms) {
  if (plan == nullptr || count == nullptr || capacity < 0 ||
      (capacity > 0 && (candidates == nullptr || ms == nullptr))) {
    return ASC_SB_INVALID_ARGUMENT;
  }
  *count = plan->tuned_count;
  for (int i = 0; i < plan->tuned_count && i < capacity; ++i) {
    candidates[i] = plan->tuned_candidate[i];
    ms[i] = plan->tuned_ms[i];
  }
  return ASC_SB_OK;
}

int asc_sb_plan_autotune(asc_sb_context* ctx, asc_sb_plan* plan, const asc_sb_vector* x,
                         const asc_sb_vector* y, int32_t count, const int32_t* variants,
                         const int32_t* lanes, int32_t reps, float* ms) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  if (plan == nullptr || count < 1 || variants == nullptr || lanes == nullptr || reps < 1) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "autotune arguments are invalid"));
  }
  for (int i = 0; i < count; ++i) {
    if (!ValidVariant(variants[i], variants[i] == ASC_SB_VARIANT_VECTOR ? lanes[i] : 1)) {
      return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "autotune names an unknown variant"));
    }
  }
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (!guard.ok()) return Finish(ctx, Fail(ASC_SB_UNAVAILABLE, "CUDA device is unavailable"));
  CompatOperands ops;
  s = ValidateCompat(ctx, &plan->matrix, x, y, &ops);
  if (!s.ok()) return Finish(ctx, s);
  if (plan->matrix.rows == 0) return Finish(ctx, Status::Ok());
  const ascb_csr a = AsCsr(plan->matrix, false);
  const int dtype = Dtype(plan->matrix.element_kind);
  cudaEvent_t start = nullptr, stop = nullptr;
  cudaError_t e = cudaEventCreate(&start);
  if (e == cudaSuccess) e = cudaEventCreate(&stop);
  int best = -1;
  float best_ms = 0.0f;
  for (int i = 0; i < count && e == cudaSuccess && s.ok(); ++i) {
    Choice c;
    c.variant = variants[i];
    c.lanes = lanes[i];
    // one warm-up, then `reps` timed products y = A x
    s = RunCsr(ctx, c, ASCB_COMPAT, a, dtype, 1.0, 0.0, AsVec(*x), AsVec(*y), nullptr,
               &plan->part);
    if (s.ok()) e = cudaEventRecord(start, ctx->stream);
    for (int r = 0; r < reps && s.ok() && e == cudaSuccess; ++r) {
      s = RunCsr(ctx, c, ASCB_COMPAT, a, dtype, 1.0, 0.0, AsVec(*x), AsVec(*y), nullptr,
                 &plan->part);
    }
    if (s.ok() && e == cudaSuccess) e = cudaEventRecord(stop, ctx->stream);
    if (s.ok() && e == cudaSuccess) e = cudaEventSynchronize(stop);
    float t = 0.0f;
    if (s.ok() && e == cudaSuccess) e = cudaEventElapsedTime(&t, start, stop);
    t /= static_cast<float>(reps);
    if (ms != nullptr) ms[i] = t;
    if (s.ok() && e == cudaSuccess && (best < 0 || t < best_ms)) {
      best = i;
      best_ms = t;
    }
  }
  if (start != nullptr) (void)cudaEventDestroy(start);
  if (stop != nullptr) (void)cudaEventDestroy(stop);
  if (!s.ok()) return Finish(ctx, s);
  if (e != cudaSuccess) {
    (void)cudaStreamSynchronize(ctx->stream);
    (void)cudaGetLastError();
    return Finish(ctx, {ASC_SB_PROVIDER,
                        std::string("CUDA failed while autotuning: ") + cudaGetErrorString(e)});
  }
  plan->variant = variants[best];
  plan->lanes = lanes[best];
  return Finish(ctx, Status::Ok());
}

int asc_sb_matrix_features(asc_sb_context* ctx, const asc_sb_sparse* m, float* features,
                           void* scratch) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (m == nullptr || features == nullptr || scratch == nullptr) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "feature arguments cannot be null"));
  }
  SparseBytes mb;
  s = ascb::host::ValidateSparse(*m, ctx->device, &mb);
  if (!s.ok()) return Finish(ctx, s);
  const ascb_csr a = AsCsr(*m, m->format == ASC_SB_CSC);
  return Finish(ctx, Launched(ctx,
                              ascb_matrix_features(
                                  ctx->stream, &a,
                                  static_cast<int>(ascb::host::ElementBytes(m->element_kind)),
                                  static_cast<unsigned long long*>(scratch), features,
                                  ctx->sm_count),
                              "CUDA could not launch the feature kernels"));
}

int asc_sb_selector_forward(asc_sb_context* ctx, int32_t n_variants, const float* params,
                            const float* x, int64_t batch, float* hidden, float* y) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (n_variants < 1 || n_variants > kSelMaxOutputs || batch < 0 ||
      (batch > 0 && (params == nullptr || x == nullptr || hidden == nullptr || y == nullptr))) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "selector forward arguments are invalid"));
  }
  return Finish(ctx, Launched(ctx, ascb_mlp_forward(ctx->stream, n_variants, params, x, batch,
                                                    hidden, y),
                              "CUDA could not launch the selector forward kernels"));
}

int asc_sb_selector_backward(asc_sb_context* ctx, int32_t n_variants, const float* params,
                             const float* x, int64_t batch, const float* hidden, const float* y,
                             const float* target, float* grads, float* loss, float* scratch) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (n_variants < 1 || n_variants > kSelMaxOutputs || batch < 0 ||
      (batch > 0 && (params == nullptr || x == nullptr || hidden == nullptr || y == nullptr ||
                     target == nullptr || grads == nullptr || scratch == nullptr))) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "selector backward arguments are invalid"));
  }
  return Finish(ctx, Launched(ctx,
                              ascb_mlp_backward(ctx->stream, n_variants, params, x, batch, hidden,
                                                y, target, grads, loss, scratch),
                              "CUDA could not launch the selector backward kernels"));
}

int asc_sb_selector_adam(asc_sb_context* ctx, float* params, const float* grads, float* m,
                         float* v, int64_t n, float lr, float beta1, float beta2, float eps,
                         int32_t step) {
  Status s = ValidateContext(ctx);
  if (!s.ok()) return Finish(ctx, s);
  std::lock_guard<std::mutex> lock(ctx->mutex);
  DeviceGuard guard(ctx->device);
  if (n < 0 || step < 1 ||
      (n > 0 && (params == nullptr || grads == nullptr || m == nullptr || v == nullptr))) {
    return Finish(ctx, Fail(ASC_SB_INVALID_ARGUMENT, "Adam arguments are invalid"));
  }
  return Finish(ctx, Launched(ctx,
                              ascb_adam_step(ctx->stream, params, grads, m, v, n, lr, beta1,
                                             beta2, eps, step),
                              "CUDA could not launch the Adam kernel"));
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
  view->stager = &ctx->stager;
  view->allocator = &ctx->allocator;
  return true;
}

}  // namespace ascb::host
