// Row-group SpMM, C += alpha * A * B with row-major B and C, sm_100a.
//
// A CSR SpMM reads one row of B per stored entry; on CUDA cores the load
// path, not HBM, is then the limit (each entry's B row crosses the L1 data
// stage again even when it hits).  Neighbouring rows of grid and stencil
// matrices share most of their columns, so this kernel processes R rows at a
// time: a plan merges the R rows' column lists once into "runs" -- one per
// distinct column, with the set of rows (a bit mask) that hold it and their
// values in row order -- and the kernel loads each B row once per run and
// applies it to every row of the mask from registers.  A warp is R rows x
// L = 32/R lanes; lane (i, l) keeps row i's accumulators for J 16-byte chunks
// of a k-tile of L*J chunks.  Each row still visits its entries in stored
// (column) order, so the EXACT form -- C(o,j) = C(o,j) + (alpha*v)*B(c,j),
// every product and sum rounded -- is the reference's per-entry update bit for
// bit (include/asc/sparse/blas.h:1736-1748); FAST uses FMA and applies alpha
// once.
//
// Plan layout (ascb_row_groups_layout): group_runs[groups+1] (first run of
// each group), run_col[nnz], run_mask[nnz], run_off[nnz] (a run's first value,
// relative to the group's first entry), vals[nnz] (the group's values sorted
// by column, then row), plus build scratch.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// ---- build -------------------------------------------------------------------

// Entry e (row r, column c) of group g = r / R: its position in the group's
// (column, row) order = entries of the group's other rows with a smaller
// column (or the same column and a smaller row) + e's position in its row.
__global__ void __launch_bounds__(kThreads)
group_rank_kernel(int64_t rows, int R, const int64_t* __restrict__ ptr,
                  const int64_t* __restrict__ idx, const int64_t* __restrict__ row_of,
                  int64_t nnz, int64_t* __restrict__ perm) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < nnz;
       e += step) {
    const int64_t r = __ldg(row_of + e);
    const int64_t c = __ldg(idx + e);
    const int64_t r0 = r / R * R;
    const int64_t r1 = r0 + R < rows ? r0 + R : rows;
    int64_t rank = e - __ldg(ptr + r);
    for (int64_t q = r0; q < r1; ++q) {
      if (q == r) continue;
      // entries of row q before column c (q > r) or at or before it (q < r)
      int64_t lo = __ldg(ptr + q), hi = __ldg(ptr + q + 1);
      while (lo < hi) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        const int64_t v = __ldg(idx + mid);
        if (v < c || (q < r && v == c)) {
          lo = mid + 1;
        } else {
          hi = mid;
        }
      }
      rank += lo - __ldg(ptr + q);
    }
    perm[__ldg(ptr + r0) + rank] = e;
  }
}

// flags[p] = 1 where position p starts a run (a group's first entry, or a
// column change).
__global__ void __launch_bounds__(kThreads)
group_flag_kernel(int R, const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                  const int64_t* __restrict__ row_of, const int64_t* __restrict__ perm,
                  int64_t nnz, int64_t* __restrict__ flags) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += step) {
    const int64_t e = __ldg(perm + p);
    const int64_t g0 = __ldg(row_of + e) / R * R;
    int64_t f = 1;
    if (p > __ldg(ptr + g0)) f = __ldg(idx + __ldg(perm + p - 1)) != __ldg(idx + e) ? 1 : 0;
    flags[p] = f;
  }
}

// Per-block sums, their exclusive scan (one block), and the final exclusive
// scan: out[p] = sum of flags before p, out[n] = total.
constexpr int kScanItems = 2048;
__global__ void __launch_bounds__(kThreads)
scan_sums_kernel(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t part[kWarps];
  const int64_t b0 = static_cast<int64_t>(blockIdx.x) * kScanItems;
  int64_t s = 0;
  for (int64_t i = b0 + threadIdx.x; i < b0 + kScanItems && i < n; i += kThreads) s += in[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kWarps; ++w) t += part[w];
    sums[blockIdx.x] = t;
  }
}
__global__ void scan_block_sums_kernel(int64_t* __restrict__ sums, int64_t blocks) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int64_t run = 0;
  for (int64_t b = 0; b < blocks; ++b) {
    const int64_t v = sums[b];
    sums[b] = run;
    run += v;
  }
  sums[blocks] = run;
}
__global__ void __launch_bounds__(kThreads)
scan_final_kernel(const int64_t* __restrict__ in, int64_t n, const int64_t* __restrict__ sums,
                  int64_t* __restrict__ out) {
  __shared__ int64_t warp_total[kWarps];
  const int64_t b0 = static_cast<int64_t>(blockIdx.x) * kScanItems;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t carry = sums[blockIdx.x];
  // kScanItems / kThreads rounds of kThreads consecutive items
  for (int64_t base = b0; base < b0 + kScanItems; base += kThreads) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < n ? in[i] : 0;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane == 31) warp_total[warp] = x;
    __syncthreads();
    int64_t before = 0, total = 0;
    for (int w = 0; w < kWarps; ++w) {
      const int64_t t = warp_total[w];
      if (w < warp) before += t;
      total += t;
    }
    if (i < n) out[i] = carry + before + x - v;
    carry += total;
    __syncthreads();
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

// Runs: column, row mask and first value of each run; values in run order.
template <typename T>
__global__ void __launch_bounds__(kThreads)
group_runs_kernel(int R, const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                  const T* __restrict__ val, const int64_t* __restrict__ row_of,
                  const int64_t* __restrict__ perm, const int64_t* __restrict__ flags,
                  const int64_t* __restrict__ run_of, int64_t nnz,
                  int64_t* __restrict__ run_col, unsigned* __restrict__ run_mask,
                  unsigned* __restrict__ run_off, T* __restrict__ vals) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz;
       p += step) {
    const int64_t e = __ldg(perm + p);
    const int64_t r = __ldg(row_of + e);
    const int64_t g0 = r / R * R;
    // run_of = exclusive scan of the run starts: a start is run run_of[p],
    // any other position belongs to the run before
    const int64_t run = __ldg(run_of + p) + __ldg(flags + p) - 1;
    vals[p] = __ldg(val + e);
    atomicOr(run_mask + run, 1u << static_cast<unsigned>(r - g0));
    if (__ldg(flags + p) != 0) {
      run_col[run] = __ldg(idx + e);
      run_off[run] = static_cast<unsigned>(p - __ldg(ptr + g0));
    }
  }
}

// group_runs[g] = runs before group g's first entry (g = 0 .. groups).
__global__ void __launch_bounds__(kThreads)
group_ptr_kernel(int64_t rows, int R, const int64_t* __restrict__ ptr,
                 const int64_t* __restrict__ run_of, int64_t groups,
                 int64_t* __restrict__ group_runs) {
  const int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g > groups) return;
  const int64_t r = g * R < rows ? g * R : rows;
  group_runs[g] = __ldg(run_of + __ldg(ptr + r));
}

// ---- product -----------------------------------------------------------------

template <typename T>
struct V16;
template <>
struct V16<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ static void split(const float4& v, float (&e)[4]) {
    e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
  }
  __device__ static float4 join(const float (&e)[4]) { return make_float4(e[0], e[1], e[2], e[3]); }
};
template <>
struct V16<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ static void split(const double2& v, double (&e)[2]) {
    e[0] = v.x; e[1] = v.y;
  }
  __device__ static double2 join(const double (&e)[2]) { return make_double2(e[0], e[1]); }
};

template <typename T, int R, int J, bool EXACT>
__global__ void __launch_bounds__(kThreads)
spmm_groups_kernel(int64_t rows, int64_t chunks, const int64_t* __restrict__ ptr,
                   const int64_t* __restrict__ group_runs, const int64_t* __restrict__ run_col,
                   const unsigned* __restrict__ run_mask, const unsigned* __restrict__ run_off,
                   const T* __restrict__ vals, const T* __restrict__ b, int64_t ldb,
                   T* __restrict__ c, int64_t ldc, T alpha) {
  using W = V16<T>;
  using V = typename W::type;
  constexpr int N = W::n;
  constexpr int L = 32 / R;            // lanes per row
  constexpr int64_t kTile = L * J;     // chunks per k-tile
  const int lane = threadIdx.x & 31;
  const int ri = lane / L;             // row within the group
  const int li = lane % L;
  const unsigned below = (1u << ri) - 1u;
  const int64_t groups = (rows + R - 1) / R;
  const int64_t tiles = (chunks + kTile - 1) / kTile;
  const int64_t items = groups * tiles;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x) >> 5;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kWarps;
  for (int64_t item = warp; item < items; item += warps) {
    const int64_t g = item / tiles;
    const int64_t tile = item - g * tiles;
    const int64_t r = g * R + ri;
    const bool row_ok = r < rows;
    T acc[J][N];
    bool live[J];
#pragma unroll
    for (int t = 0; t < J; ++t) {
      const int64_t ch = tile * kTile + t * L + li;
      live[t] = row_ok && ch < chunks;
      if (EXACT && live[t]) {
        W::split(*reinterpret_cast<const V*>(c + r * ldc + ch * N), acc[t]);
      } else {
#pragma unroll
        for (int e = 0; e < N; ++e) acc[t][e] = T(0);
      }
    }
    const int64_t first = __ldg(ptr + g * R);
    const int64_t rb = __ldg(group_runs + g), re = __ldg(group_runs + g + 1);
    for (int64_t run = rb; run < re; ++run) {
      const unsigned mask = __ldg(run_mask + run);
      if (((mask >> ri) & 1u) == 0u) continue;
      const int64_t col = __ldg(run_col + run);
      const T v = __ldg(vals + first + __ldg(run_off + run) + __popc(mask & below));
      const T av = EXACT ? mul_rn(alpha, v) : v;
      V bv[J];
#pragma unroll
      for (int t = 0; t < J; ++t) {
        const int64_t ch = tile * kTile + t * L + li;
        bv[t] = live[t] ? __ldg(reinterpret_cast<const V*>(b + col * ldb + ch * N)) : V{};
      }
#pragma unroll
      for (int t = 0; t < J; ++t) {
        T e[N];
        W::split(bv[t], e);
#pragma unroll
        for (int i = 0; i < N; ++i) {
          acc[t][i] = EXACT ? add_rn(acc[t][i], mul_rn(av, e[i])) : fma(av, e[i], acc[t][i]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < J; ++t) {
      if (!live[t]) continue;
      const int64_t ch = tile * kTile + t * L + li;
      V* cp = reinterpret_cast<V*>(c + r * ldc + ch * N);
      if (EXACT) {
        *cp = W::join(acc[t]);
      } else {
        T old[N];
        W::split(*cp, old);
#pragma unroll
        for (int i = 0; i < N; ++i) acc[t][i] = fma(alpha, acc[t][i], old[i]);
        *cp = W::join(acc[t]);
      }
    }
  }
}

unsigned grid(int64_t work, int sm) {
  const int64_t needed = (work + kThreads - 1) / kThreads;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * 8;
  return static_cast<unsigned>(needed < 1 ? 1 : (needed < cap ? needed : cap));
}

template <typename T, int R, int J>
int launch_groups(cudaStream_t s, bool exact, const ascb_csr* a, const ascb_row_groups* rg,
                  int64_t chunks, const void* b, int64_t ldb, void* c, int64_t ldc, T alpha,
                  int sm) {
  constexpr int L = 32 / R;
  const int64_t groups = (a->rows + R - 1) / R;
  const int64_t tiles = (chunks + L * J - 1) / (L * J);
  const int64_t warps = groups * tiles;
  const int64_t needed = (warps + kWarps - 1) / kWarps;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * 8;
  const unsigned blocks = static_cast<unsigned>(needed < 1 ? 1 : (needed < cap ? needed : cap));
  const auto* vals = static_cast<const T*>(rg->vals);
  if (exact) {
    spmm_groups_kernel<T, R, J, true><<<blocks, kThreads, 0, s>>>(
        a->rows, chunks, a->ptr, rg->group_runs, rg->run_col, rg->run_mask, rg->run_off, vals,
        static_cast<const T*>(b), ldb, static_cast<T*>(c), ldc, alpha);
  } else {
    spmm_groups_kernel<T, R, J, false><<<blocks, kThreads, 0, s>>>(
        a->rows, chunks, a->ptr, rg->group_runs, rg->run_col, rg->run_mask, rg->run_off, vals,
        static_cast<const T*>(b), ldb, static_cast<T*>(c), ldc, alpha);
  }
  return static_cast<int>(cudaGetLastError());
}

// Lanes per row L = 32 / R; chunks per lane J: the k-tile L*J covers the
// row's chunks where it can (fewer passes over the runs), at most 8 chunks per
// lane (registers).
template <typename T>
int groups_typed(cudaStream_t s, bool exact, const ascb_csr* a, const ascb_row_groups* rg,
                 int64_t chunks, const void* b, int64_t ldb, void* c, int64_t ldc, double alpha,
                 int sm) {
  const T al = static_cast<T>(alpha);
#define ASCB_GROUPS(RR, JJ) \
  return launch_groups<T, RR, JJ>(s, exact, a, rg, chunks, b, ldb, c, ldc, al, sm)
  const int64_t L = 32 / rg->rows_per_group;
  const int64_t per_lane = (chunks + L - 1) / L;
  switch (rg->rows_per_group) {
    case 32:
      if (per_lane <= 1) ASCB_GROUPS(32, 1);
      if (per_lane <= 2) ASCB_GROUPS(32, 2);
      if (per_lane <= 4) ASCB_GROUPS(32, 4);
      ASCB_GROUPS(32, 8);
    case 16:
      if (per_lane <= 1) ASCB_GROUPS(16, 1);
      if (per_lane <= 2) ASCB_GROUPS(16, 2);
      if (per_lane <= 4) ASCB_GROUPS(16, 4);
      ASCB_GROUPS(16, 8);
    case 8:
      if (per_lane <= 1) ASCB_GROUPS(8, 1);
      if (per_lane <= 2) ASCB_GROUPS(8, 2);
      if (per_lane <= 4) ASCB_GROUPS(8, 4);
      ASCB_GROUPS(8, 8);
    case 4:
      if (per_lane <= 1) ASCB_GROUPS(4, 1);
      if (per_lane <= 2) ASCB_GROUPS(4, 2);
      if (per_lane <= 4) ASCB_GROUPS(4, 4);
      ASCB_GROUPS(4, 8);
    default:
      if (per_lane <= 1) ASCB_GROUPS(2, 1);
      if (per_lane <= 2) ASCB_GROUPS(2, 2);
      if (per_lane <= 4) ASCB_GROUPS(2, 4);
      ASCB_GROUPS(2, 8);
  }
#undef ASCB_GROUPS
}

}  // namespace
}  // namespace ascb

extern "C" {

ascb_row_groups_layout ascb_row_groups_layout_for(int64_t rows, int64_t nnz, int elem_bytes) {
  ascb_row_groups_layout l{};
  const size_t n = static_cast<size_t>(nnz > 0 ? nnz : 1);
  const size_t groups = static_cast<size_t>(rows / 2 + 2);  // the most groups: R = 2
  size_t at = 0;
  l.group_runs = at;
  at += ascb::up256(groups * 8);
  l.run_col = at;
  at += ascb::up256(n * 8);
  l.run_mask = at;
  at += ascb::up256(n * 4);
  l.run_off = at;
  at += ascb::up256(n * 4);
  l.vals = at;
  at += ascb::up256(n * static_cast<size_t>(elem_bytes));
  l.persistent = at;
  // build scratch: row of each entry, permutation, run starts, run ids (+1),
  // block sums
  l.row_of = at;
  at += ascb::up256(n * 8);
  l.perm = at;
  at += ascb::up256(n * 8);
  l.flags = at;
  at += ascb::up256(n * 8);
  l.run_of = at;
  at += ascb::up256((n + 1) * 8);
  l.sums = at;
  at += ascb::up256((n / ascb::kScanItems + 2) * 8);
  l.total = at;
  return l;
}

int ascb_row_groups_build(void* stream, const ascb_csr* a, int elem_bytes, int rows_per_group,
                          void* base, ascb_row_groups* out, int sm_count) {
  const ascb_row_groups_layout l = ascb_row_groups_layout_for(a->rows, a->nnz, elem_bytes);
  auto* p = static_cast<unsigned char*>(base);
  auto s = static_cast<cudaStream_t>(stream);
  const int R = rows_per_group;
  out->rows_per_group = R;
  out->group_runs = reinterpret_cast<int64_t*>(p + l.group_runs);
  out->run_col = reinterpret_cast<int64_t*>(p + l.run_col);
  out->run_mask = reinterpret_cast<unsigned*>(p + l.run_mask);
  out->run_off = reinterpret_cast<unsigned*>(p + l.run_off);
  out->vals = p + l.vals;
  const int64_t nnz = a->nnz;
  const int64_t groups = (a->rows + R - 1) / R;
  auto* row_of = reinterpret_cast<int64_t*>(p + l.row_of);
  auto* perm = reinterpret_cast<int64_t*>(p + l.perm);
  auto* flags = reinterpret_cast<int64_t*>(p + l.flags);
  auto* run_of = reinterpret_cast<int64_t*>(p + l.run_of);
  auto* sums = reinterpret_cast<int64_t*>(p + l.sums);
  int rc = ascb_outer_of_entries(stream, a->ptr, a->rows, row_of, sm_count);
  if (rc != 0) return rc;
  cudaError_t e = cudaMemsetAsync(out->run_mask, 0, static_cast<size_t>(nnz > 0 ? nnz : 1) * 4, s);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (nnz > 0) {
    ascb::group_rank_kernel<<<ascb::grid(nnz, sm_count), ascb::kThreads, 0, s>>>(
        a->rows, R, a->ptr, a->idx, row_of, nnz, perm);
    ascb::group_flag_kernel<<<ascb::grid(nnz, sm_count), ascb::kThreads, 0, s>>>(
        R, a->ptr, a->idx, row_of, perm, nnz, flags);
    const int64_t blocks = (nnz + ascb::kScanItems - 1) / ascb::kScanItems;
    ascb::scan_sums_kernel<<<static_cast<unsigned>(blocks), ascb::kThreads, 0, s>>>(flags, nnz,
                                                                                  sums);
    ascb::scan_block_sums_kernel<<<1, 32, 0, s>>>(sums, blocks);
    ascb::scan_final_kernel<<<static_cast<unsigned>(blocks), ascb::kThreads, 0, s>>>(
        flags, nnz, sums, run_of);
    if (elem_bytes == 8) {
      ascb::group_runs_kernel<double><<<ascb::grid(nnz, sm_count), ascb::kThreads, 0, s>>>(
          R, a->ptr, a->idx, static_cast<const double*>(a->val), row_of, perm, flags, run_of,
          nnz, out->run_col, out->run_mask, out->run_off, static_cast<double*>(out->vals));
    } else {
      ascb::group_runs_kernel<float><<<ascb::grid(nnz, sm_count), ascb::kThreads, 0, s>>>(
          R, a->ptr, a->idx, static_cast<const float*>(a->val), row_of, perm, flags, run_of,
          nnz, out->run_col, out->run_mask, out->run_off, static_cast<float*>(out->vals));
    }
  } else {
    e = cudaMemsetAsync(run_of, 0, 8, s);
    if (e != cudaSuccess) return static_cast<int>(e);
  }
  ascb::group_ptr_kernel<<<static_cast<unsigned>((groups + 1 + ascb::kThreads - 1) /
                                                  ascb::kThreads),
                           ascb::kThreads, 0, s>>>(a->rows, R, a->ptr, run_of, groups,
                                                   out->group_runs);
  return static_cast<int>(cudaGetLastError());
}

int ascb_scan_i64(void* stream, const int64_t* in, int64_t n, int64_t* out, int64_t* sums) {
  if (n <= 0) {
    return static_cast<int>(cudaMemsetAsync(out, 0, 8, static_cast<cudaStream_t>(stream)));
  }
  auto s = static_cast<cudaStream_t>(stream);
  const int64_t blocks = (n + ascb::kScanItems - 1) / ascb::kScanItems;
  ascb::scan_sums_kernel<<<static_cast<unsigned>(blocks), ascb::kThreads, 0, s>>>(in, n, sums);
  ascb::scan_block_sums_kernel<<<1, 32, 0, s>>>(sums, blocks);
  ascb::scan_final_kernel<<<static_cast<unsigned>(blocks), ascb::kThreads, 0, s>>>(in, n, sums,
                                                                                 out);
  return static_cast<int>(cudaGetLastError());
}

int ascb_spmm_groups(void* stream, int dtype, int exact, const ascb_csr* a,
                     const ascb_row_groups* rg, int64_t k, const void* b, int64_t ldb, void* c,
                     int64_t ldc, double alpha, int sm_count) {
  if (a->rows <= 0 || k <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return ascb::groups_typed<double>(s, exact != 0, a, rg, k / 2, b, ldb, c, ldc, alpha,
                                      sm_count);
  }
  return ascb::groups_typed<float>(s, exact != 0, a, rg, k / 4, b, ldb, c, ldc, alpha, sm_count);
}

}  // extern "C"
