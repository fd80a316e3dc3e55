// TMA-staged SpMM, C += alpha * A * B with row-major B and C, sm_100a.
//
// A CSR SpMM reads one row of B per stored entry.  Neighbouring rows of grid
// and stencil matrices share most of their columns, and the columns of a few
// consecutive rows form a handful of contiguous runs (a 27-point stencil: 9
// runs of R + 2 columns for R rows).  A plan (ascb_staged_build) cuts the
// rows into groups -- 16 rows, and wide groups of 32 and 64 rows that merge
// the columns two or four 16-row groups share -- and records, per group, its
// distinct columns as "slots" in column order, the maximal runs of
// consecutive columns among them ("segments"), and per stored entry the slot
// of its column (16 bits).
//
// The kernel runs a two-stage TMA pipeline per CTA over stages of NG
// consecutive groups: while it computes stage s, one warp has the bulk copies
// of stage s+1 in flight -- every segment's rows of B (one cp.async.bulk per
// segment when ldb == k), the stage's row offsets, values and entry slots,
// and its rows of C when they are long -- completing on the stage's mbarrier;
// that warp reads the tables that place the copies two stages ahead.
// Compute reads only shared memory: G lanes own a row's 16-byte chunks of C
// and walk its entries in stored order, each entry one shared-memory vector
// load of B(slot, chunk).  So B crosses L2 -> SM once per group and slot
// instead of once per entry, and no load waits on global memory during
// compute (but for short rows of C).
//
// Arithmetic per entry, in stored order:
//   EXACT: C(o,j) = C(o,j) + (alpha*v)*B(c,j), every product and sum rounded
//          (the reference's per-entry update, include/asc/sparse/blas.h:
//          1736-1748; bit-exact);
//   FAST:  acc = fma(v, B(c,j), acc), then C(o,j) = fma(alpha, acc, C(o,j)).
// Stage waits are bounded: a wait that gives up records 1 in *status, waits
// (bounded) for the copies it issued, and the CTA stops.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;
constexpr int kGroupRows = 16;           // rows per group
constexpr int kLevels = 3;               // groups of 16, 32 and 64 rows
constexpr uint32_t kWaitLimit = 1u << 20;
constexpr uint32_t kSuspendNs = tma::kTmaSuspendNs;  // stage-wait suspend hint
constexpr int kUnroll = 4;

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

unsigned grid_for(int64_t work, int sm) {
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * 8;
  const int64_t b = (work + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 1 ? 1 : (b < cap ? b : cap));
}

// ---- build -------------------------------------------------------------------
// Inputs: the row groups of R = 16 (ascb_row_groups_build) and their build
// scratch -- per sorted position p (group, column, row order): perm[p] (the
// stored entry), flags[p] (1 where a run starts), run_of[p] (runs before p).

// slot of every stored entry; segment starts among the runs.
__global__ void __launch_bounds__(kThreads)
staged_slot_kernel(const int64_t* __restrict__ row_of, const int64_t* __restrict__ perm,
                   const int64_t* __restrict__ flags, const int64_t* __restrict__ run_of,
                   const int64_t* __restrict__ group_runs, const int64_t* __restrict__ run_col,
                   int64_t nnz, uint16_t* __restrict__ slot, int64_t* __restrict__ seg_flag) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += step) {
    const int64_t e = __ldg(perm + p);
    const int64_t g = __ldg(row_of + e) / kGroupRows;
    const int64_t f = __ldg(flags + p);
    const int64_t run = __ldg(run_of + p) + f - 1;
    const int64_t first = __ldg(group_runs + g);
    const int64_t rel = run - first;
    slot[e] = static_cast<uint16_t>(rel < 65535 ? rel : 65535);
    if (f != 0) {
      seg_flag[run] =
          (run == first || __ldg(run_col + run - 1) + 1 != __ldg(run_col + run)) ? 1 : 0;
    }
  }
}

// segment s: first column and first run (runs are numbered over all groups
// in order, so run - group_runs[g0] is its slot in a stage starting at g0).
__global__ void __launch_bounds__(kThreads)
staged_seg_kernel(const int64_t* __restrict__ flags, const int64_t* __restrict__ run_of,
                  const int64_t* __restrict__ run_col, const int64_t* __restrict__ seg_flag,
                  const int64_t* __restrict__ seg_of, int64_t nnz, int64_t* __restrict__ seg_col,
                  int64_t* __restrict__ seg_run) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += step) {
    if (__ldg(flags + p) == 0) continue;
    const int64_t run = __ldg(run_of + p);
    if (__ldg(seg_flag + run) == 0) continue;
    const int64_t s = __ldg(seg_of + run);
    seg_col[s] = __ldg(run_col + run);
    seg_run[s] = run;
  }
}

// seg_len[s] = runs up to the next segment's first run (the groups' runs are
// consecutive, so the last segment of a group ends where the next group
// starts); segs and runs are read from the finished tables.
__global__ void __launch_bounds__(kThreads)
staged_len_kernel(const int64_t* __restrict__ seg_run, const int64_t* __restrict__ group_segs,
                  const int64_t* __restrict__ group_runs, int64_t groups,
                  int32_t* __restrict__ seg_len) {
  const int64_t segs = __ldg(group_segs + groups);
  const int64_t runs = __ldg(group_runs + groups);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < segs;
       s += step) {
    const int64_t next = s + 1 < segs ? __ldg(seg_run + s + 1) : runs;
    seg_len[s] = static_cast<int32_t>(next - __ldg(seg_run + s));
  }
}

// group_segs[g] = segments before group g (g = 0 .. groups).
__global__ void __launch_bounds__(kThreads)
staged_group_kernel(const int64_t* __restrict__ group_runs, const int64_t* __restrict__ seg_of,
                    int64_t groups, int64_t* __restrict__ group_segs) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g > groups) return;
  group_segs[g] = __ldg(seg_of + __ldg(group_runs + g));
}

// Largest slot and entry counts over the aligned windows of 1, 2, 4, ...
// groups of `group_rows` rows (`windows` widths: the stage widths).
__global__ void __launch_bounds__(kThreads)
staged_caps_kernel(const int64_t* __restrict__ ptr, int64_t rows, int64_t group_rows,
                   const int64_t* __restrict__ group_runs, int64_t groups, int windows,
                   unsigned long long* __restrict__ caps) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < groups;
       g += step) {
    for (int w = 0; w < windows; ++w) {
      const int64_t ng = int64_t{1} << w;
      if (g % ng != 0) continue;
      const int64_t ge = g + ng < groups ? g + ng : groups;
      const int64_t r0 = g * group_rows;
      const int64_t r1 = ge * group_rows < rows ? ge * group_rows : rows;
      atomicMax(caps + 2 * w, static_cast<unsigned long long>(__ldg(group_runs + ge) -
                                                              __ldg(group_runs + g)));
      atomicMax(caps + 2 * w + 1,
                static_cast<unsigned long long>(__ldg(ptr + r1) - __ldg(ptr + r0)));
    }
  }
}

// ---- wide groups: M = 2 or 4 consecutive 16-row groups merged ------------------
// A wide group (rows 16 M w .. 16 M (w + 1) - 1) holds the distinct columns of
// its M groups, in column order; segments are its maximal runs of consecutive
// columns.  Built from the 16-row tables: a run is its column's FIRST in the
// wide group unless an earlier group of the wide group holds that column; the
// wide slot of a run is the number of distinct columns below its column,
// summed over the M groups from prefix counts F of the first-flags.

// group of run u: the g with group_runs[g] <= u < group_runs[g + 1]
__device__ __forceinline__ int64_t group_of_run(const int64_t* __restrict__ group_runs,
                                                int64_t groups, int64_t u) {
  int64_t lo = 0, hi = groups - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(group_runs + mid) <= u) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}
// first position in run_col[lo, hi) (increasing) whose column is >= c
__device__ __forceinline__ int64_t lower_col(const int64_t* __restrict__ run_col, int64_t lo,
                                             int64_t hi, int64_t c) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(run_col + mid) < c) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads)
wide_first_kernel(const int64_t* __restrict__ group_runs, const int64_t* __restrict__ run_col,
                  int64_t groups, int64_t merge, int64_t nnz, int64_t* __restrict__ first) {
  const int64_t runs = __ldg(group_runs + groups);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < nnz;
       u += step) {
    if (u >= runs) break;
    const int64_t g = group_of_run(group_runs, groups, u);
    const int64_t c = __ldg(run_col + u);
    int64_t f = 1;
    for (int64_t h = g / merge * merge; h < g; ++h) {
      const int64_t lo = __ldg(group_runs + h), hi = __ldg(group_runs + h + 1);
      const int64_t q = lower_col(run_col, lo, hi, c);
      if (q < hi && __ldg(run_col + q) == c) f = 0;
    }
    first[u] = f;
  }
}

// wide slot of every run; merged column table (first runs only)
__global__ void __launch_bounds__(kThreads)
wide_rank_kernel(const int64_t* __restrict__ group_runs, const int64_t* __restrict__ run_col,
                 const int64_t* __restrict__ first, const int64_t* __restrict__ fsum,
                 int64_t groups, int64_t merge, int64_t nnz,
                 int32_t* __restrict__ wide_slot_of, int64_t* __restrict__ wide_col) {
  const int64_t runs = __ldg(group_runs + groups);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; u < nnz;
       u += step) {
    if (u >= runs) break;
    const int64_t g = group_of_run(group_runs, groups, u);
    const int64_t c = __ldg(run_col + u);
    const int64_t w0 = g / merge * merge;
    const int64_t w1 = w0 + merge < groups ? w0 + merge : groups;
    int64_t r = 0;
    for (int64_t h = w0; h < w1; ++h) {
      const int64_t lo = __ldg(group_runs + h), hi = __ldg(group_runs + h + 1);
      const int64_t q = h == g ? u : lower_col(run_col, lo, hi, c);
      r += __ldg(fsum + q) - __ldg(fsum + lo);
    }
    wide_slot_of[u] = static_cast<int32_t>(r < 65535 ? r : 65535);
    if (__ldg(first + u) != 0) wide_col[__ldg(fsum + __ldg(group_runs + w0)) + r] = c;
  }
}

// wide_runs[w] = merged slots before wide group w (w = 0 .. wide groups)
__global__ void __launch_bounds__(kThreads)
wide_group_kernel(const int64_t* __restrict__ group_runs, const int64_t* __restrict__ fsum,
                  int64_t groups, int64_t merge, int64_t wide,
                  int64_t* __restrict__ wide_runs) {
  const int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w > wide) return;
  const int64_t g = w * merge < groups ? w * merge : groups;
  wide_runs[w] = __ldg(fsum + __ldg(group_runs + g));
}

// wide slot of every stored entry
__global__ void __launch_bounds__(kThreads)
wide_entry_kernel(const int64_t* __restrict__ ptr, int64_t rows,
                  const int64_t* __restrict__ group_runs, const uint16_t* __restrict__ slot,
                  const int32_t* __restrict__ wide_slot_of, uint16_t* __restrict__ wide_slot) {
  // one warp per 16-row group's rows, entries strided over the lanes
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5);
       r < rows; r += warps) {
    const int64_t base = __ldg(group_runs + r / kGroupRows);
    const int64_t e1 = __ldg(ptr + r + 1);
    for (int64_t e = __ldg(ptr + r) + lane; e < e1; e += 32) {
      const uint16_t s = __ldg(slot + e);  // 65535: the group overflowed its slots
      wide_slot[e] = s == 65535 ? s : static_cast<uint16_t>(__ldg(wide_slot_of + base + s));
    }
  }
}

// segment starts over the merged columns: a column break or a wide group's
// first slot (the second pass sets the latter)
__global__ void __launch_bounds__(kThreads)
wide_break_kernel(const int64_t* __restrict__ wide_col, const int64_t* __restrict__ wide_runs,
                  int64_t wide, int64_t nnz, int64_t* __restrict__ flag) {
  const int64_t total = __ldg(wide_runs + wide);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
       i += step) {
    if (i >= total) break;
    flag[i] = (i == 0 || __ldg(wide_col + i - 1) + 1 != __ldg(wide_col + i)) ? 1 : 0;
  }
}
__global__ void __launch_bounds__(kThreads)
wide_start_kernel(const int64_t* __restrict__ wide_runs, int64_t wide, int64_t* __restrict__ flag) {
  const int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= wide) return;
  const int64_t i = __ldg(wide_runs + w);
  if (i < __ldg(wide_runs + w + 1)) flag[i] = 1;
}
__global__ void __launch_bounds__(kThreads)
wide_seg_kernel(const int64_t* __restrict__ wide_col, const int64_t* __restrict__ wide_runs,
                int64_t wide, const int64_t* __restrict__ flag, const int64_t* __restrict__ seg_of,
                int64_t nnz, int64_t* __restrict__ seg_col, int64_t* __restrict__ seg_run) {
  const int64_t total = __ldg(wide_runs + wide);
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
       i += step) {
    if (i >= total) break;
    if (__ldg(flag + i) == 0) continue;
    const int64_t s = __ldg(seg_of + i);
    seg_col[s] = __ldg(wide_col + i);
    seg_run[s] = i;
  }
}

// ---- product -----------------------------------------------------------------

template <typename T>
struct Vec;
template <>
struct Vec<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ static void split(const float4& v, float (&e)[4]) {
    e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
  }
  __device__ static float4 join(const float (&e)[4]) { return make_float4(e[0], e[1], e[2], e[3]); }
};
template <>
struct Vec<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ static void split(const double2& v, double (&e)[2]) {
    e[0] = v.x; e[1] = v.y;
  }
  __device__ static double2 join(const double (&e)[2]) { return make_double2(e[0], e[1]); }
};

// Rows of C of more than 8 chunks (128 bytes; G >= 16 lanes per row) arrive
// with the stage's copies instead of one global load per row (27-point 128^3
// stencil, FP32, B200: k = 128 2.77 -> 2.09 ms; k = 8 and 32 0.246 / 0.494 ->
// 0.253 / 0.501 ms, the stage's extra shared memory costing more than the
// load it saves).
__host__ __device__ constexpr bool stage_c(int64_t chunks) { return chunks > 8; }

// Byte layout of one stage for `slots` B rows of `chunks` 16-byte chunks and
// `entries` stored entries of NG groups.
constexpr int kMaxStageGroups = 16;
struct StageHeader {  // written by the producer before it releases the stage
  int64_t r0, r1, z0;
  int32_t lead_p, lead_v, lead_s, pad;
  int64_t slots[kMaxStageGroups + 1];  // group_runs of the stage's groups, from g0
};
struct StageLayout {
  uint32_t b, c, ptr, val, slot, hdr, bar, bytes;
};
template <typename T>
__host__ __device__ StageLayout stage_layout(int64_t slots, int64_t chunks, int64_t entries,
                                             int ng, int64_t group_rows) {
  StageLayout l;
  size_t at = 0;
  l.b = 0;
  at += static_cast<size_t>(slots * chunks) * 16;
  l.c = static_cast<uint32_t>(at);  // the stage's rows of C (stage_c(chunks), ldc == k)
  if (stage_c(chunks)) at += static_cast<size_t>(ng) * group_rows * chunks * 16;
  l.ptr = static_cast<uint32_t>(at);
  at += ((static_cast<size_t>(ng) * group_rows + 4) * 8 + 15) / 16 * 16;
  l.val = static_cast<uint32_t>(at);
  at += ((static_cast<size_t>(entries) + 16 / sizeof(T) * 2) * sizeof(T) + 15) / 16 * 16;
  l.slot = static_cast<uint32_t>(at);
  at += ((static_cast<size_t>(entries) + 16) * 2 + 15) / 16 * 16;
  l.hdr = static_cast<uint32_t>(at);
  at += (sizeof(StageHeader) + 15) / 16 * 16;
  l.bar = static_cast<uint32_t>(at);
  at += 16;  // full, empty
  l.bytes = static_cast<uint32_t>((at + 127) / 128 * 128);
  return l;
}

struct StagedArgs {
  int64_t rows, nnz, groups, chunks;
  const int64_t* ptr;
  const void* val;
  const uint16_t* slot;
  const int64_t* group_runs;  // slots before each group
  const int64_t* group_segs;
  const int64_t* seg_col;
  const int64_t* seg_run;
  const int32_t* seg_len;
  const void* b;
  int64_t ldb;
  void* c;
  int64_t ldc;
  int ng;           // groups per stage
  int group_shift;  // log2 of the rows per group (16, 32 or 64)
  StageLayout lay;
  int* status;
};

constexpr int kConsumerWarps = kThreads / 32;
constexpr int kAllThreads = kThreads + 32;  // + the producer warp

__device__ __forceinline__ void mbar_init_n(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(tma::smem_addr(bar)),
               "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;\n" ::"r"(tma::smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive1(uint64_t* bar) {
  asm volatile(
      "{\n .reg .b64 st;\n"
      " mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(tma::smem_addr(bar))
      : "memory");
}

// Warp 8 produces: for each of the CTA's stages (s = blockIdx.x, + gridDim.x,
// ...) it waits for the buffer's `empty` barrier, writes the stage header,
// announces the byte count on `full`, issues the bulk copies (one per B
// segment, lanes in parallel; the A arrays by lane 0), loads the few tail
// elements a rounded copy would overrun, and arrives on `full`.  Warps 0-7
// consume: wait `full`, compute the stage's rows from shared memory, arrive
// on `empty`.  G lanes per row (a power of two, <= 32), J chunks per lane.
// Every wait is bounded; a role that gives up sets *status and the shared
// abort flag, which ends the other role's waits.
template <typename T, int G, int J, bool EXACT>
__global__ void __launch_bounds__(kAllThreads)
spmm_staged_kernel(StagedArgs a, T alpha) {
  using namespace tma;
  using W = Vec<T>;
  using V = typename W::type;
  constexpr int N = W::n;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int abort_flag;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int64_t stages = (a.groups + a.ng - 1) / a.ng;
  const int64_t first = blockIdx.x;
  if (first >= stages) return;
  const int64_t stride = gridDim.x;
  const T* val = static_cast<const T*>(a.val);
  const T* bmat = static_cast<const T*>(a.b);
  T* cmat = static_cast<T*>(a.c);
  auto stage_at = [&](int b) { return smem + static_cast<size_t>(b) * a.lay.bytes; };
  auto full_of = [&](int b) { return reinterpret_cast<uint64_t*>(stage_at(b) + a.lay.bar); };
  auto empty_of = [&](int b) { return full_of(b) + 1; };
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init_n(full_of(b), 1);
      mbar_init_n(empty_of(b), kConsumerWarps);
    }
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    for (uint32_t n = 0; n < kWaitLimit; ++n) {
      if (mbar_try_wait(bar, parity, kSuspendNs)) return true;
      if (*reinterpret_cast<volatile int*>(&abort_flag) != 0) return false;
    }
    return false;
  };
  auto give_up = [&]() {
    *reinterpret_cast<volatile int*>(&abort_flag) = 1;
    if (a.status != nullptr) atomicOr(a.status, 1);
  };
  const int64_t row_bytes = a.chunks * 16;
  // long, contiguous rows of C arrive with each stage's copies
  // (G >= 16 exactly when chunks > 8: the kernels for fewer lanes per row
  // carry no shared-memory C path)
  const bool c_staged =
      G >= 16 && a.ldc == a.chunks * (16 / static_cast<int64_t>(sizeof(T)));

  if (warp == kConsumerWarps) {
    // ---------------- producer ----------------
    // Table reads run ahead of the copies: a stage's extent and group tables
    // are loaded two stages early, its first 32 segments one stage early, so
    // no stage waits on a chain of dependent global loads.
    struct Extent {
      int64_t z0, z1, s0, s1, gslot;
    };
    struct Segs {
      int64_t run, col, len;
    };
    auto extent_of = [&](int64_t s, Extent& m) {
      if (s >= stages) return;
      const int64_t g0 = s * a.ng;
      const int64_t g1 = g0 + a.ng < a.groups ? g0 + a.ng : a.groups;
      const int64_t r0 = g0 << a.group_shift;
      const int64_t r1 = (g1 << a.group_shift) < a.rows ? (g1 << a.group_shift) : a.rows;
      m.z0 = __ldg(a.ptr + r0);
      m.z1 = __ldg(a.ptr + r1);
      m.s0 = __ldg(a.group_segs + g0);
      m.s1 = __ldg(a.group_segs + g1);
      m.gslot = lane <= g1 - g0 ? __ldg(a.group_runs + g0 + lane) : 0;
    };
    auto segs_of = [&](int64_t s, const Extent& m, Segs& g) {
      const int64_t q = m.s0 + lane;
      if (s >= stages || q >= m.s1) return;
      g.run = __ldg(a.seg_run + q);
      g.col = __ldg(a.seg_col + q);
      g.len = __ldg(a.seg_len + q);
    };
    Extent cur{}, nxt{}, far{};
    Segs cur_seg{}, nxt_seg{};
    extent_of(first, cur);
    extent_of(first + stride, nxt);
    segs_of(first, cur, cur_seg);
    int64_t i = 0;
    for (int64_t s = first; s < stages; s += stride, ++i) {
      segs_of(s + stride, nxt, nxt_seg);
      extent_of(s + 2 * stride, far);
      const int b = static_cast<int>(i & 1);
      if (i >= 2 && !wait(empty_of(b), static_cast<uint32_t>(((i >> 1) - 1) & 1))) {
        if (lane == 0) give_up();
        break;
      }
      unsigned char* base = stage_at(b);
      auto* hdr = reinterpret_cast<StageHeader*>(base + a.lay.hdr);
      const int64_t g0 = s * a.ng;
      const int64_t g1 = g0 + a.ng < a.groups ? g0 + a.ng : a.groups;
      const int64_t r0 = g0 << a.group_shift;
      const int64_t r1 = (g1 << a.group_shift) < a.rows ? (g1 << a.group_shift) : a.rows;
      const int64_t z0 = cur.z0, z1 = cur.z1, s0 = cur.s0, s1 = cur.s1, gslot = cur.gslot;
      const int64_t slot0 = __shfl_sync(0xffffffffu, gslot, 0);
      const int64_t slots = __shfl_sync(0xffffffffu, gslot, static_cast<int>(g1 - g0)) - slot0;
      const CopyPlan<8> cp = plan_copy<8>(r0, r1 - r0 + 1, a.rows + 1);
      const CopyPlan<sizeof(T)> cv = plan_copy<sizeof(T)>(z0, z1 - z0, a.nnz);
      const CopyPlan<2> cs = plan_copy<2>(z0, z1 - z0, a.nnz);
      if (lane <= g1 - g0) hdr->slots[lane] = gslot;
      if (lane == 0) {
        hdr->r0 = r0;
        hdr->r1 = r1;
        hdr->z0 = z0;
        hdr->lead_p = cp.lead;
        hdr->lead_v = cv.lead;
        hdr->lead_s = cs.lead;
      }
      // this warp's earlier generic stores into the buffer (tails of its
      // last use) come before the bulk copies that overwrite them
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        const uint32_t cbytes = c_staged ? static_cast<uint32_t>((r1 - r0) * row_bytes) : 0u;
        mbar_expect(full_of(b), cp.bytes + cv.bytes + cs.bytes + cbytes +
                                    static_cast<uint32_t>(slots * row_bytes));
        if (cbytes) bulk_g2s(base + a.lay.c, cmat + r0 * a.ldc, cbytes, full_of(b));
        if (cp.bytes) bulk_g2s(base + a.lay.ptr, a.ptr + cp.g0, cp.bytes, full_of(b));
        if (cv.bytes) bulk_g2s(base + a.lay.val, val + cv.g0, cv.bytes, full_of(b));
        if (cs.bytes) bulk_g2s(base + a.lay.slot, a.slot + cs.g0, cs.bytes, full_of(b));
      }
      __syncwarp();
      for (int64_t q = s0 + lane; q < s1; q += 32) {
        Segs g = cur_seg;  // the first 32 segments were loaded a stage ago
        if (q >= s0 + 32) {
          g.run = __ldg(a.seg_run + q);
          g.col = __ldg(a.seg_col + q);
          g.len = __ldg(a.seg_len + q);
        }
        const int64_t slot = g.run - slot0;
        unsigned char* dst = base + a.lay.b + slot * row_bytes;
        if (a.ldb == a.chunks * (16 / static_cast<int64_t>(sizeof(T)))) {
          bulk_g2s(dst, bmat + g.col * a.ldb, static_cast<uint32_t>(g.len * row_bytes),
                   full_of(b));
        } else {
          for (int64_t r = 0; r < g.len; ++r) {
            bulk_g2s(dst + r * row_bytes, bmat + (g.col + r) * a.ldb,
                     static_cast<uint32_t>(row_bytes), full_of(b));
          }
        }
      }
      cur = nxt;
      nxt = far;
      cur_seg = nxt_seg;
      // plain-load tails at the ends of the arrays
      auto* sptr = reinterpret_cast<int64_t*>(base + a.lay.ptr) + cp.lead;
      auto* sval = reinterpret_cast<T*>(base + a.lay.val) + cv.lead;
      auto* sslot = reinterpret_cast<uint16_t*>(base + a.lay.slot) + cs.lead;
      if (lane < cp.tail) sptr[cp.tail0 - r0 + lane] = __ldg(a.ptr + cp.tail0 + lane);
      if (lane < cv.tail) sval[cv.tail0 - z0 + lane] = __ldg(val + cv.tail0 + lane);
      if (lane < cs.tail) sslot[cs.tail0 - z0 + lane] = __ldg(a.slot + cs.tail0 + lane);
      __syncwarp();
      if (lane == 0) mbar_arrive1(full_of(b));
    }
    // every copy this warp issued has landed before the CTA ends (bounded,
    // and regardless of the abort flag)
    if (lane == 0) {
      const int64_t issued = i;
      for (int64_t k = issued > 2 ? issued - 2 : 0; k < issued; ++k) {
        for (uint32_t n = 0; n < kWaitLimit; ++n) {
          if (mbar_try_wait(full_of(static_cast<int>(k & 1)), static_cast<uint32_t>((k >> 1) & 1),
                            kSuspendNs)) {
            break;
          }
        }
      }
    }
  } else {
    // ---------------- consumers ----------------
    const int lc = tid % G;
    int64_t i = 0;
    for (int64_t s = first; s < stages; s += stride, ++i) {
      const int b = static_cast<int>(i & 1);
      if (!wait(full_of(b), static_cast<uint32_t>((i >> 1) & 1))) {
        if (lane == 0) give_up();
        break;
      }
      const unsigned char* base = stage_at(b);
      const auto* hdr = reinterpret_cast<const StageHeader*>(base + a.lay.hdr);
      const int64_t r0 = hdr->r0;
      const int64_t z0 = hdr->z0;
      const int nrows = static_cast<int>(hdr->r1 - r0);
      const int64_t slot0 = hdr->slots[0];
      const auto* sptr = reinterpret_cast<const int64_t*>(base + a.lay.ptr) + hdr->lead_p;
      const auto* sval = reinterpret_cast<const T*>(base + a.lay.val) + hdr->lead_v;
      const auto* sslot = reinterpret_cast<const uint16_t*>(base + a.lay.slot) + hdr->lead_s;
      // 32-bit shared-memory byte offsets: this lane's first chunk of slot 0
      const uint32_t rbytes = static_cast<uint32_t>(row_bytes);
      const unsigned char* sbb = base + a.lay.b + static_cast<uint32_t>(lc) * 16u;
      const unsigned char* scb = base + a.lay.c;
      for (int rl = tid / G; rl < nrows; rl += kThreads / G) {
        const int pb = static_cast<int>(sptr[rl] - z0);
        const int pe = static_cast<int>(sptr[rl + 1] - z0);
        if (pb == pe) continue;  // C unchanged in both forms
        const unsigned char* rowb =
            sbb + static_cast<uint32_t>(hdr->slots[rl >> a.group_shift] - slot0) * rbytes;
        T* crow = cmat + (r0 + rl) * a.ldc;
        T acc[J][N];
        bool live[J];
#pragma unroll
        for (int t = 0; t < J; ++t) {
          const int64_t ch = lc + static_cast<int64_t>(t) * G;
          live[t] = ch < a.chunks;
          if (EXACT && live[t]) {
            W::split(c_staged ? *reinterpret_cast<const V*>(scb + (rl * a.chunks + ch) * 16)
                              : *reinterpret_cast<const V*>(crow + ch * N),
                     acc[t]);
          } else {
#pragma unroll
            for (int e = 0; e < N; ++e) acc[t][e] = T(0);
          }
        }
        int q = pb;
        for (; q + kUnroll <= pe; q += kUnroll) {
          T av[kUnroll];
          uint32_t sl[kUnroll];
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
            av[u] = EXACT ? mul_rn(alpha, sval[q + u]) : sval[q + u];
            sl[u] = static_cast<uint32_t>(sslot[q + u]) * rbytes;
          }
          V bv[kUnroll][J];
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int t = 0; t < J; ++t) {
              bv[u][t] = live[t] ? *reinterpret_cast<const V*>(rowb + sl[u] + t * G * 16) : V{};
            }
          }
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int t = 0; t < J; ++t) {
              T e[N];
              W::split(bv[u][t], e);
#pragma unroll
              for (int k = 0; k < N; ++k) {
                acc[t][k] = EXACT ? add_rn(acc[t][k], mul_rn(av[u], e[k]))
                                  : fma(av[u], e[k], acc[t][k]);
              }
            }
          }
        }
        for (; q < pe; ++q) {
          const T av = EXACT ? mul_rn(alpha, sval[q]) : sval[q];
          const uint32_t sl = static_cast<uint32_t>(sslot[q]) * rbytes;
#pragma unroll
          for (int t = 0; t < J; ++t) {
            if (!live[t]) continue;
            T e[N];
            W::split(*reinterpret_cast<const V*>(rowb + sl + t * G * 16), e);
#pragma unroll
            for (int k = 0; k < N; ++k) {
              acc[t][k] = EXACT ? add_rn(acc[t][k], mul_rn(av, e[k])) : fma(av, e[k], acc[t][k]);
            }
          }
        }
#pragma unroll
        for (int t = 0; t < J; ++t) {
          if (!live[t]) continue;
          const int64_t ch = lc + static_cast<int64_t>(t) * G;
          V* cpv = reinterpret_cast<V*>(crow + ch * N);
          if (!EXACT) {
            T old[N];
            W::split(c_staged ? *reinterpret_cast<const V*>(scb + (rl * a.chunks + ch) * 16) : *cpv,
                     old);
#pragma unroll
            for (int k = 0; k < N; ++k) acc[t][k] = fma(alpha, acc[t][k], old[k]);
          }
          *cpv = W::join(acc[t]);
        }
      }
      // this warp is done with the buffer
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) mbar_arrive1(empty_of(b));
    }
  }
  __syncthreads();
}

// CTAs per SM for one instantiation and dynamic shared-memory size (opt-in
// set once per device and size).
template <typename Kernel>
int prepare(Kernel kernel, size_t smem, int* per_sm) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return static_cast<int>(e);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kernel, kAllThreads, smem);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (*per_sm < 1) return static_cast<int>(cudaErrorInvalidConfiguration);
  return 0;
}

template <typename T, int G, int J>
int launch_staged(cudaStream_t s, bool exact, const StagedArgs& args, T alpha, int sm) {
  const size_t smem = static_cast<size_t>(args.lay.bytes) * 2;
  auto kernel = exact ? spmm_staged_kernel<T, G, J, true> : spmm_staged_kernel<T, G, J, false>;
  int per_sm = 0;
  const int rc = prepare(kernel, smem, &per_sm);
  if (rc != 0) return rc;
  const int64_t stages = (args.groups + args.ng - 1) / args.ng;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * per_sm;
  const unsigned blocks = static_cast<unsigned>(stages < cap ? stages : cap);
  kernel<<<blocks, kAllThreads, smem, s>>>(args, alpha);
  return static_cast<int>(cudaGetLastError());
}

// G = min(32, chunks) rounded up to a power of two, J = ceil(chunks / G) <= 4.
template <typename T>
int staged_typed(cudaStream_t s, bool exact, const StagedArgs& args, double alpha, int sm) {
  const T al = static_cast<T>(alpha);
  const int64_t ch = args.chunks;
#define ASCB_STAGED(GG, JJ) return launch_staged<T, GG, JJ>(s, exact, args, al, sm)
  if (ch <= 1) ASCB_STAGED(1, 1);
  if (ch <= 2) ASCB_STAGED(2, 1);
  if (ch <= 4) ASCB_STAGED(4, 1);
  if (ch <= 8) ASCB_STAGED(8, 1);
  if (ch <= 16) ASCB_STAGED(16, 1);
  if (ch <= 32) ASCB_STAGED(32, 1);
  if (ch <= 64) ASCB_STAGED(32, 2);
  ASCB_STAGED(32, 4);
#undef ASCB_STAGED
}

}  // namespace
}  // namespace ascb

extern "C" {

ascb_staged_layout ascb_staged_layout_for(int64_t rows, int64_t nnz) {
  ascb_staged_layout l{};
  const size_t n = static_cast<size_t>(nnz > 0 ? nnz : 1);
  size_t at = 0;
  // the tables of one level (groups of 16 rows, then wide groups of 32, 64)
  auto level = [&](ascb_staged_level_layout& v, size_t group_rows) {
    const size_t groups = static_cast<size_t>(rows) / group_rows + 2;
    v.group_runs = at;
    at += ascb::up256((groups + 1) * 8);
    v.group_segs = at;
    at += ascb::up256((groups + 1) * 8);
    v.seg_col = at;
    at += ascb::up256(n * 8);
    v.seg_run = at;
    at += ascb::up256(n * 8);
    v.seg_len = at;
    at += ascb::up256(n * 4);
    v.slot = at;
    at += ascb::up256(n * 2);
    v.caps = at;
    at += 256;
  };
  for (int v = 0; v < ascb::kLevels; ++v) level(l.level[v], size_t{ascb::kGroupRows} << v);
  l.persistent = at;
  l.seg_flag = at;  // build scratch
  at += ascb::up256((n + 1) * 8);
  l.seg_of = at;
  at += ascb::up256((n + 2) * 8);
  l.sums = at;
  at += ascb::up256((n / 2048 + 2) * 8);
  l.wide_slot_of = at;
  at += ascb::up256(n * 4);
  l.wide_col = at;
  at += ascb::up256(n * 8);
  l.total = at;
  return l;
}

int ascb_staged_build(void* stream, const ascb_csr* a, const ascb_row_groups* rg16,
                      const void* groups_base, int elem_bytes, void* base,
                      ascb_staged_spmm* levels, int sm_count) {
  if (rg16->rows_per_group != ascb::kGroupRows) return static_cast<int>(cudaErrorInvalidValue);
  auto s = static_cast<cudaStream_t>(stream);
  const ascb_staged_layout l = ascb_staged_layout_for(a->rows, a->nnz);
  const ascb_row_groups_layout gl = ascb_row_groups_layout_for(a->rows, a->nnz, elem_bytes);
  auto* p = static_cast<unsigned char*>(base);
  const auto* gp = static_cast<const unsigned char*>(groups_base);
  const auto* row_of = reinterpret_cast<const int64_t*>(gp + gl.row_of);
  const auto* perm = reinterpret_cast<const int64_t*>(gp + gl.perm);
  const auto* flags = reinterpret_cast<const int64_t*>(gp + gl.flags);
  const auto* run_of = reinterpret_cast<const int64_t*>(gp + gl.run_of);
  const int64_t nnz = a->nnz;
  auto tables = [&](ascb_staged_spmm* t, const ascb_staged_level_layout& v, int64_t group_rows) {
    t->group_rows = group_rows;
    t->groups = (a->rows + group_rows - 1) / group_rows;
    t->group_runs = reinterpret_cast<int64_t*>(p + v.group_runs);
    t->group_segs = reinterpret_cast<int64_t*>(p + v.group_segs);
    t->seg_col = reinterpret_cast<int64_t*>(p + v.seg_col);
    t->seg_run = reinterpret_cast<int64_t*>(p + v.seg_run);
    t->seg_len = reinterpret_cast<int32_t*>(p + v.seg_len);
    t->slot = reinterpret_cast<uint16_t*>(p + v.slot);
    t->caps = reinterpret_cast<unsigned long long*>(p + v.caps);
  };
  for (int v = 0; v < ascb::kLevels; ++v) {
    tables(levels + v, l.level[v], int64_t{ascb::kGroupRows} << v);
  }
  ascb_staged_spmm* out = levels;
  const int64_t groups = out->groups;
  auto* seg_flag = reinterpret_cast<int64_t*>(p + l.seg_flag);
  auto* seg_of = reinterpret_cast<int64_t*>(p + l.seg_of);
  auto* sums = reinterpret_cast<int64_t*>(p + l.sums);
  auto* wide_slot_of = reinterpret_cast<int32_t*>(p + l.wide_slot_of);
  auto* wide_col = reinterpret_cast<int64_t*>(p + l.wide_col);
  const size_t flag_bytes = static_cast<size_t>(nnz + 1) * 8;
  cudaError_t e = cudaMemcpyAsync(out->group_runs, rg16->group_runs,
                                  static_cast<size_t>(groups + 1) * 8, cudaMemcpyDeviceToDevice, s);
  for (int v = 0; v < ascb::kLevels && e == cudaSuccess; ++v) {
    e = cudaMemsetAsync(levels[v].caps, 0, 256, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(seg_flag, 0, flag_bytes, s);
  if (e != cudaSuccess) return static_cast<int>(e);
  const unsigned g = ascb::grid_for(nnz, sm_count);
  const unsigned kt = ascb::kThreads;
  auto blocks_for = [&](int64_t n) { return static_cast<unsigned>((n + kt - 1) / kt); };
  // ---- groups of 16 rows
  if (nnz > 0) {
    ascb::staged_slot_kernel<<<g, kt, 0, s>>>(row_of, perm, flags, run_of, rg16->group_runs,
                                              rg16->run_col, nnz, out->slot, seg_flag);
    // segments before each run (exclusive scan over nnz + 1 >= runs + 1 entries)
    int rc = ascb_scan_i64(stream, seg_flag, nnz + 1, seg_of, sums);
    if (rc != 0) return rc;
    ascb::staged_seg_kernel<<<g, kt, 0, s>>>(flags, run_of, rg16->run_col, seg_flag, seg_of, nnz,
                                             out->seg_col, out->seg_run);
  } else {
    e = cudaMemsetAsync(seg_of, 0, 16, s);
    if (e != cudaSuccess) return static_cast<int>(e);
  }
  ascb::staged_group_kernel<<<blocks_for(groups + 1), kt, 0, s>>>(out->group_runs, seg_of,
                                                                  groups, out->group_segs);
  if (nnz > 0) {
    ascb::staged_len_kernel<<<g, kt, 0, s>>>(out->seg_run, out->group_segs, out->group_runs,
                                             groups, out->seg_len);
  }
  ascb::staged_caps_kernel<<<ascb::grid_for(groups, sm_count), kt, 0, s>>>(
      a->ptr, a->rows, ascb::kGroupRows, out->group_runs, groups, 5, out->caps);
  // ---- wide groups of 16 M rows (M = 2, 4), from the 16-row tables
  for (int v = 1; v < ascb::kLevels; ++v) {
    ascb_staged_spmm* wide = levels + v;
    const int64_t merge = int64_t{1} << v;
    const int64_t wgroups = wide->groups;
    if (nnz > 0) {
      e = cudaMemsetAsync(seg_flag, 0, flag_bytes, s);
      if (e != cudaSuccess) return static_cast<int>(e);
      ascb::wide_first_kernel<<<g, kt, 0, s>>>(out->group_runs, rg16->run_col, groups, merge, nnz,
                                               seg_flag);
      int rc = ascb_scan_i64(stream, seg_flag, nnz + 1, seg_of, sums);  // F
      if (rc != 0) return rc;
      ascb::wide_rank_kernel<<<g, kt, 0, s>>>(out->group_runs, rg16->run_col, seg_flag, seg_of,
                                              groups, merge, nnz, wide_slot_of, wide_col);
      ascb::wide_group_kernel<<<blocks_for(wgroups + 1), kt, 0, s>>>(
          out->group_runs, seg_of, groups, merge, wgroups, wide->group_runs);
      ascb::wide_entry_kernel<<<ascb::grid_for(a->rows * 32, sm_count), kt, 0, s>>>(
          a->ptr, a->rows, out->group_runs, out->slot, wide_slot_of, wide->slot);
      // segments of the merged columns
      e = cudaMemsetAsync(seg_flag, 0, flag_bytes, s);
      if (e != cudaSuccess) return static_cast<int>(e);
      ascb::wide_break_kernel<<<g, kt, 0, s>>>(wide_col, wide->group_runs, wgroups, nnz,
                                               seg_flag);
      ascb::wide_start_kernel<<<blocks_for(wgroups), kt, 0, s>>>(wide->group_runs, wgroups,
                                                                 seg_flag);
      rc = ascb_scan_i64(stream, seg_flag, nnz + 1, seg_of, sums);
      if (rc != 0) return rc;
      ascb::wide_seg_kernel<<<g, kt, 0, s>>>(wide_col, wide->group_runs, wgroups, seg_flag,
                                             seg_of, nnz, wide->seg_col, wide->seg_run);
    } else {
      e = cudaMemsetAsync(wide->group_runs, 0, static_cast<size_t>(wgroups + 1) * 8, s);
      if (e == cudaSuccess) e = cudaMemsetAsync(seg_of, 0, 16, s);
      if (e != cudaSuccess) return static_cast<int>(e);
    }
    ascb::staged_group_kernel<<<blocks_for(wgroups + 1), kt, 0, s>>>(wide->group_runs, seg_of,
                                                                     wgroups, wide->group_segs);
    if (nnz > 0) {
      ascb::staged_len_kernel<<<g, kt, 0, s>>>(wide->seg_run, wide->group_segs,
                                               wide->group_runs, wgroups, wide->seg_len);
    }
    ascb::staged_caps_kernel<<<ascb::grid_for(wgroups, sm_count), kt, 0, s>>>(
        a->ptr, a->rows, wide->group_rows, wide->group_runs, wgroups, 5, wide->caps);
  }
  return static_cast<int>(cudaGetLastError());
}

size_t ascb_staged_stage_bytes(int dtype, int64_t k, int64_t slots, int64_t entries, int ng,
                               int64_t group_rows) {
  const int64_t chunks = k * (dtype == ASCB_F64 ? 8 : 4) / 16;
  return dtype == ASCB_F64
             ? ascb::stage_layout<double>(slots, chunks, entries, ng, group_rows).bytes
             : ascb::stage_layout<float>(slots, chunks, entries, ng, group_rows).bytes;
}

int ascb_staged_groups_per_stage(int dtype, int64_t k, int64_t group_rows) {
  const int64_t chunks = k * (dtype == ASCB_F64 ? 8 : 4) / 16;
  int g = 1;
  while (g < 32 && g < chunks) g <<= 1;
  const int64_t ng = ascb::kThreads / g / group_rows;  // one consumer pass
  return ng < 1 ? 1 : static_cast<int>(ng);
}

int ascb_spmm_staged(void* stream, int dtype, int exact, const ascb_csr* a,
                     const ascb_staged_spmm* st, int64_t k, const void* b, int64_t ldb, void* c,
                     int64_t ldc, double alpha, int64_t max_slots, int64_t max_entries,
                     int* status, int sm_count) {
  if (a->rows <= 0 || k <= 0) return 0;
  int shift = 0;
  while (shift < 8 && (int64_t{1} << shift) < st->group_rows) ++shift;
  if (st->group_rows < ascb::kGroupRows || (int64_t{1} << shift) != st->group_rows ||
      st->group_rows > (int64_t{ascb::kGroupRows} << (ascb::kLevels - 1))) {
    return static_cast<int>(cudaErrorInvalidValue);
  }
  ascb::StagedArgs args{};
  args.rows = a->rows;
  args.nnz = a->nnz;
  args.groups = st->groups;
  args.chunks = k * (dtype == ASCB_F64 ? 8 : 4) / 16;
  args.ptr = a->ptr;
  args.val = a->val;
  args.slot = st->slot;
  args.group_runs = st->group_runs;
  args.group_segs = st->group_segs;
  args.seg_col = st->seg_col;
  args.seg_run = st->seg_run;
  args.seg_len = st->seg_len;
  args.b = b;
  args.ldb = ldb;
  args.c = c;
  args.ldc = ldc;
  args.ng = ascb_staged_groups_per_stage(dtype, k, st->group_rows);
  args.group_shift = shift;
  args.status = status;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    args.lay = ascb::stage_layout<double>(max_slots, args.chunks, max_entries, args.ng,
                                          st->group_rows);
    return ascb::staged_typed<double>(s, exact != 0, args, alpha, sm_count);
  }
  args.lay =
      ascb::stage_layout<float>(max_slots, args.chunks, max_entries, args.ng, st->group_rows);
  return ascb::staged_typed<float>(s, exact != 0, args, alpha, sm_count);
}

}  // extern "C"
