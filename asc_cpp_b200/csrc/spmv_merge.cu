// Merge-based, TMA-fed CSR SpMV for sm_100a.
//
// Work split.  The plan partitions the rows into tiles of kItems merge items
// (one item per row end plus one per nonzero; the row-aligned partition of
// row_tile_kernel with weight 1) and records, per tile boundary, the pair
// (first row, ptr[first row]).  A warp owns a contiguous range of tiles.
//
// Per tile, one lane issues three TMA bulk copies (cp.async.bulk) into the
// warp's shared-memory stage -- the tile's row offsets, its column indices and
// its values -- completing on an mbarrier.  The copies for tile t+1 are in
// flight while the warp computes tile t, so streaming costs no LSU issue slots
// and only the x gathers sit on the critical path.
//
// Compute (round 0 = the tile's first kItems merge items):
//   A. lanes walk the staged nonzeros with unit stride, gather x through the
//      read-only path and overwrite each value slot with its product;
//   B. lane k consumes merge items [8k, 8k+8) in order (found by a merge-path
//      search over the staged row offsets): a nonzero adds its product to the
//      running row sum, a row end emits the row.  Every lane does the same
//      amount of work whatever the row-length distribution;
//   C. sums of rows that cross lane boundaries are joined:
//        FAST  -- a segmented warp scan of the lanes' open partial sums;
//        EXACT -- the running sum is handed lane to lane in stored order, so
//                 every row is summed exactly as the serial reference does.
// The tile's last row may be longer than the tile (a long row); its remainder
// is summed by the whole warp after round 0.
//
// EXACT reproduces the reference bit for bit:
//   compat   (src/sparse/reference_blas.cc:13-39): s = +0, s = s + v*x, ...,
//            y = alpha*s (+ beta*y)
//   standard (include/asc/sparse/blas.h:1653-1665): s = y, s = s + (alpha*v)*x
// FAST forms plain sums and reassociates them at lane boundaries; its error is
// within gamma_{n+2}(|alpha||A||x| + |beta||y|).
//
// Waits on the mbarriers are bounded: a wait that gives up records an error
// in the caller's status word, waits once more (also bounded) for the copy it
// issued, and the warp returns.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kThreads = kWarpsPerCta * 32;
constexpr int kItems = 256;              // merge items per tile (round 0)
constexpr int kPerLane = kItems / 32;    // merge items per lane
constexpr int kPad = 4;                  // alignment slack, elements
constexpr int kStages = 2;
constexpr uint32_t kWaitLimit = 1u << 20;  // polls before a wait gives up
constexpr uint32_t kSuspendNs = tma::kTmaSuspendNs;  // stage-wait suspend hint
constexpr int kMaxDevices = 64;

// Every TMA destination starts on a 16-byte boundary; each array has room for
// the copy's alignment lead and rounding (at most 3 elements each side).
template <typename T>
struct alignas(16) Stage {
  alignas(16) int64_t ptr[kItems + 2 + kPad];  // row offsets ptr[R0 .. R1]
  alignas(16) int64_t idx[kItems + kPad];      // column indices of the first window
  alignas(16) T val[kItems + 2 * kPad];        // values, then products in place
  alignas(16) uint64_t bar;                    // mbarrier of this stage
};

using namespace tma;

template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T product(T alpha, T v, T xv) {
  if (EXACT && STANDARD) return mul_rn(mul_rn(alpha, v), xv);
  return EXACT ? mul_rn(v, xv) : v * xv;
}
template <bool EXACT, typename T>
__device__ __forceinline__ T add(T a, T b) {
  return EXACT ? add_rn(a, b) : a + b;
}
// Row result from its sum.  EXACT+STANDARD sums already start from y.
template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T finish(T s, T alpha, T beta, const T* yp) {
  if (EXACT) {
    if (STANDARD) return s;
    T r = mul_rn(alpha, s);
    if (beta != T(0)) r = add_rn(r, mul_rn(beta, *yp));
    return r;
  }
  if (STANDARD) return fma(alpha, s, *yp);
  return beta != T(0) ? fma(alpha, s, beta * *yp) : alpha * s;
}
template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T row_init(const T* yp) {
  return (EXACT && STANDARD) ? *yp : T(0);
}

// Tile t: rows [R0, R1), nonzeros [Z0, Z1).
struct TileInfo {
  int64_t r0, r1, z0, z1;
};

template <typename T, bool EXACT, bool STANDARD, bool UNIT>
__global__ void __launch_bounds__(kThreads)
merge_kernel(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
             const T* __restrict__ val, const T* __restrict__ x, int64_t incx,
             T* __restrict__ y, int64_t incy, T alpha, T beta,
             const int64_t* __restrict__ bounds, int64_t ntiles, int64_t rows, int64_t nnz,
             int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  Stage<T>* st = reinterpret_cast<Stage<T>*>(smem_raw) + warp * kStages;

  const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp;
  const int64_t warp_count = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  const int64_t per_warp = (ntiles + warp_count - 1) / warp_count;
  const int64_t tb = warp_id * per_warp;
  const int64_t te = tb + per_warp < ntiles ? tb + per_warp : ntiles;
  if (tb >= te) return;

  if (lane == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&st[s].bar);
    fence_mbar_init();
  }
  __syncwarp();

  auto tile_info = [&](int64_t t) {
    TileInfo ti;
    ti.r0 = __ldg(bounds + 2 * t);
    ti.z0 = __ldg(bounds + 2 * t + 1);
    ti.r1 = __ldg(bounds + 2 * t + 2);
    ti.z1 = __ldg(bounds + 2 * t + 3);
    return ti;
  };
  // Lane 0 issues the stage's three bulk copies; tails go by plain loads
  // after the wait (only near the ends of the arrays).
  auto issue = [&](const TileInfo& ti, Stage<T>& s) {
    if (lane != 0) return;
    const int64_t window = ti.z1 - ti.z0 < kItems ? ti.z1 - ti.z0 : kItems;
    const CopyPlan<8> cp = plan_copy<8>(ti.r0, ti.r1 - ti.r0 + 1, rows + 1);
    const CopyPlan<8> ci = plan_copy<8>(ti.z0, window, nnz);
    const CopyPlan<sizeof(T)> cv = plan_copy<sizeof(T)>(ti.z0, window, nnz);
    mbar_arrive_expect_tx(&s.bar, cp.bytes + ci.bytes + cv.bytes);
    if (cp.bytes) bulk_g2s(s.ptr, ptr + cp.g0, cp.bytes, &s.bar);
    if (ci.bytes) bulk_g2s(s.idx, idx + ci.g0, ci.bytes, &s.bar);
    if (cv.bytes) bulk_g2s(s.val, val + cv.g0, cv.bytes, &s.bar);
  };
  // Per-stage mbarrier phase and in-flight bits (registers, not arrays).
  uint32_t phase_bits = 0, pending_bits = 0;
  // Bounded wait for stage si.  On timeout: flag the status word, give every
  // copy this warp still has in flight one more bounded wait, and report.
  auto wait = [&](int si) -> bool {
    uint32_t n = 0;  // the loop condition is warp-uniform, so is the outcome
    while (!__all_sync(0xffffffffu, mbar_try_wait(&st[si].bar, (phase_bits >> si) & 1u, kSuspendNs))) {
      if (++n >= kWaitLimit) {
        if (lane == 0 && status != nullptr) atomicOr(status, 1);
        for (int k = 0; k < kStages; ++k) {
          if (!((pending_bits >> k) & 1u)) continue;
          for (uint32_t m = 0; m < kWaitLimit && !mbar_try_wait(&st[k].bar, (phase_bits >> k) & 1u, kSuspendNs);
               ++m) {
          }
        }
        return false;
      }
    }
    pending_bits &= ~(1u << si);
    phase_bits ^= 1u << si;
    return true;
  };

  TileInfo cur = tile_info(tb);
  issue(cur, st[0]);
  pending_bits |= 1u;

  for (int64_t t = tb; t < te; ++t) {
    const int si = static_cast<int>((t - tb) & 1);
    Stage<T>& s = st[si];
    TileInfo nxt;
    if (t + 1 < te) {
      nxt = tile_info(t + 1);
      issue(nxt, st[si ^ 1]);
      pending_bits |= 1u << (si ^ 1);
    }
    if (!wait(si)) return;

    const int nr = static_cast<int>(cur.r1 - cur.r0);
    if (nr == 0) {  // tile inside a long row that an earlier tile finishes
      cur = nxt;
      continue;
    }
    const int64_t n_nz = cur.z1 - cur.z0;
    const int window = static_cast<int>(n_nz < kItems ? n_nz : kItems);
    // element `first` of each copy sits at slot `lead` (recomputed by all)
    const int lp = static_cast<int>(cur.r0 & 1);
    const int li = static_cast<int>(cur.z0 & 1);
    const int lv = static_cast<int>(cur.z0 % (16 / sizeof(T)));
    const int64_t* sp = s.ptr + lp;
    const int64_t* si_ = s.idx + li;
    T* sv = s.val + lv;
    {  // plain-load tails at the ends of the arrays
      const CopyPlan<8> cp = plan_copy<8>(cur.r0, nr + 1, rows + 1);
      const CopyPlan<8> ci = plan_copy<8>(cur.z0, window, nnz);
      const CopyPlan<sizeof(T)> cv = plan_copy<sizeof(T)>(cur.z0, window, nnz);
      if (lane < cp.tail) const_cast<int64_t*>(sp)[cp.tail0 - cur.r0 + lane] = __ldg(ptr + cp.tail0 + lane);
      if (lane < ci.tail) const_cast<int64_t*>(si_)[ci.tail0 - cur.z0 + lane] = __ldg(idx + ci.tail0 + lane);
      if (lane < cv.tail) sv[cv.tail0 - cur.z0 + lane] = __ldg(val + cv.tail0 + lane);
      __syncwarp();
    }

    // A. products of the staged window, written over the values
    for (int q0 = 0; q0 < window; q0 += 32 * 4) {
      int64_t c[4];
      T v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u * 32 + lane;
        if (q < window) {
          c[u] = si_[q];
          v[u] = sv[q];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u * 32 + lane;
        if (q < window) sv[q] = product<EXACT, STANDARD>(alpha, v[u], ld_gather(&at<UNIT>(x, c[u], incx)));
      }
    }
    __syncwarp();

    // B. merge items [d0, d1) of round 0
    const int n0 = static_cast<int>(nr + n_nz < kItems ? nr + n_nz : kItems);
    const int d0 = lane * kPerLane < n0 ? lane * kPerLane : n0;
    const int d1 = d0 + kPerLane < n0 ? d0 + kPerLane : n0;
    int i, j;  // rows ended, nonzeros consumed (tile-local)
    {
      int lo = d0 - static_cast<int>(n_nz < d0 ? n_nz : d0);
      int hi = d0 < nr ? d0 : nr;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sp[mid + 1] - cur.z0 <= d0 - mid - 1) {
          lo = mid + 1;
        } else {
          hi = mid;
        }
      }
      i = lo;
      j = d0 - lo;
    }
    // a lane that starts inside a row continues a sum begun by earlier lanes
    const bool cont = d0 < d1 ? (i < nr && j > sp[i] - cur.z0) : true;
    int64_t row_end = i < nr ? sp[i + 1] - cur.z0 : INT64_MAX;
    T acc = T(0);
    if (!cont && i < nr) acc = row_init<EXACT, STANDARD>(&at<UNIT>(y, cur.r0 + i, incy));
    bool in_first = cont;   // still in the continued (first) segment
    bool has_end = false;
    T first_sum = T(0);     // FAST: sum of the continued segment
    int first_row = -1;     // row whose end this lane emits for the continuation
    const int j_first = j;  // EXACT: continued segment is [j_first, j_first_end)
    int j_first_end = j;
    for (int d = d0; d < d1; ++d) {
      if (j < row_end) {
        if (!(EXACT && in_first)) acc = add<EXACT>(acc, sv[j]);
        ++j;
        if (in_first) j_first_end = j;
      } else {
        T* yp = &at<UNIT>(y, cur.r0 + i, incy);
        if (in_first) {
          first_row = i;  // joined with the carry in phase C
          first_sum = acc;
          in_first = false;
        } else {
          *yp = finish<EXACT, STANDARD>(acc, alpha, beta, yp);
        }
        has_end = true;
        ++i;
        row_end = i < nr ? sp[i + 1] - cur.z0 : INT64_MAX;
        acc = i < nr ? row_init<EXACT, STANDARD>(&at<UNIT>(y, cur.r0 + i, incy)) : T(0);
      }
    }
    // acc = open sum of the row in progress at the lane's end (if in_first,
    // FAST: the lane's whole contribution to the continued row)

    // C. join the sums across lanes
    T carry_out;
    if (!EXACT) {
      T tail = in_first ? acc : acc;  // open partial of the last segment
      // segmented inclusive scan: c_k = has_end_k ? tail_k : c_{k-1} + tail_k
      T c = tail;
      bool f = has_end;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T cu = __shfl_up_sync(0xffffffffu, c, o);
        const bool fu = __shfl_up_sync(0xffffffffu, f, o);
        if (lane >= o) {
          if (!f) c = cu + c;
          f = f || fu;
        }
      }
      T carry_in = __shfl_up_sync(0xffffffffu, c, 1);
      if (lane == 0) carry_in = T(0);
      if (first_row >= 0) {
        T* yp = &at<UNIT>(y, cur.r0 + first_row, incy);
        *yp = finish<EXACT, STANDARD>(carry_in + first_sum, alpha, beta, yp);
      }
      carry_out = __shfl_sync(0xffffffffu, c, 31);
    } else {
      // exact: hand the running sum lane to lane in stored order.  Lanes past
      // the last item (only in tiles whose last row ends in round 0, so their
      // carry is never used) need nothing.
      bool resolved = !cont || d0 == d1;
      T c = acc;  // resolved lanes: carry out = open sum of own last segment
      for (int step = 0; step < 32; ++step) {
        const T cu = __shfl_up_sync(0xffffffffu, c, 1);
        const bool ru = __shfl_up_sync(0xffffffffu, resolved, 1);
        if (!resolved && (lane == 0 || ru)) {
          T sum = lane == 0 ? T(0) : cu;
          for (int q = j_first; q < j_first_end; ++q) sum = add_rn(sum, sv[q]);
          if (first_row >= 0) {
            T* yp = &at<UNIT>(y, cur.r0 + first_row, incy);
            *yp = finish<EXACT, STANDARD>(sum, alpha, beta, yp);
            c = acc;
          } else {
            c = sum;
          }
          resolved = true;
        }
        if (__all_sync(0xffffffffu, resolved)) break;
      }
      carry_out = __shfl_sync(0xffffffffu, c, 31);
    }

    // Long last row: its end item lies beyond round 0.
    const int64_t last_end_item = static_cast<int64_t>(nr - 1) + n_nz;
    if (nr > 0 && last_end_item >= n0) {
      const int jr = __shfl_sync(0xffffffffu, j, 31);  // nonzeros consumed in round 0
      const int64_t rest_begin = cur.z0 + jr;
      T* yp = &at<UNIT>(y, cur.r1 - 1, incy);
      T total;
      if (!EXACT) {
        T part = T(0);
        for (int q = jr + lane; q < window; q += 32) part += sv[q];
        for (int64_t p = cur.z0 + window + lane; p < cur.z1; p += 32) {
          part = fma(ld_stream(val + p), ld_gather(&at<UNIT>(x, ld_stream(idx + p), incx)), part);
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) part += shfl_xor(part, m);
        total = carry_out + part;
      } else {
        total = carry_out;
        if (lane == 0) {
          for (int q = jr; q < window; ++q) total = add_rn(total, sv[q]);
        }
        __syncwarp();
        for (int64_t p0 = cur.z0 + window; p0 < cur.z1; p0 += kItems) {
          const int n = static_cast<int>(cur.z1 - p0 < kItems ? cur.z1 - p0 : kItems);
          for (int q = lane; q < n; q += 32) {
            sv[q] = product<true, STANDARD>(alpha, ld_stream(val + p0 + q),
                                            ld_gather(&at<UNIT>(x, ld_stream(idx + p0 + q), incx)));
          }
          __syncwarp();
          if (lane == 0) {
            for (int q = 0; q < n; ++q) total = add_rn(total, sv[q]);
          }
          __syncwarp();
        }
        (void)rest_begin;
      }
      if (lane == 0) *yp = finish<EXACT, STANDARD>(total, alpha, beta, yp);
    }
    // This stage's shared memory was read and written by the generic proxy;
    // order that before the next TMA (async proxy) write into it.
    fence_proxy_async();
    __syncwarp();
    cur = nxt;
  }
}

template <typename T>
constexpr size_t smem_bytes() {
  return sizeof(Stage<T>) * kStages * kWarpsPerCta;
}

// Per instantiation (the Tag parameters), per device: the shared-memory
// opt-in and the resident CTAs per SM.
template <typename T, bool EXACT, bool STANDARD, bool UNIT, typename Kernel>
int configure(Kernel kernel, size_t smem, int* ctas_per_sm) {
  static int cached[kMaxDevices] = {};
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (device < 0 || device >= kMaxDevices || cached[device] == 0) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    if (n <= 0) n = 1;
    if (device >= 0 && device < kMaxDevices) cached[device] = n;
    *ctas_per_sm = n;
    return 0;
  }
  *ctas_per_sm = cached[device];
  return 0;
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT>
int launch(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
           const ascb_vec* y, const int64_t* bounds, int64_t ntiles, int sm_count, int* status) {
  auto kernel = merge_kernel<T, EXACT, STANDARD, UNIT>;
  int per_sm = 1;
  const int err = configure<T, EXACT, STANDARD, UNIT>(kernel, smem_bytes<T>(), &per_sm);
  if (err != 0) return err;
  const int64_t warps_needed = (ntiles + 1) / 2;  // at least two tiles per warp
  const int64_t ctas_needed = (warps_needed + kWarpsPerCta - 1) / kWarpsPerCta;
  const int64_t resident = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * per_sm;
  const unsigned blocks = static_cast<unsigned>(
      ctas_needed < 1 ? 1 : (ctas_needed < resident ? ctas_needed : resident));
  kernel<<<blocks, kThreads, smem_bytes<T>(), stream>>>(
      a->ptr, a->idx, static_cast<const T*>(a->val), static_cast<const T*>(x->data), x->stride,
      static_cast<T*>(y->data), y->stride, alpha, beta, bounds, ntiles, a->rows, a->nnz, status);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, bool EXACT>
int by_form(cudaStream_t s, int form, const ascb_csr* a, double alpha, double beta,
            const ascb_vec* x, const ascb_vec* y, const int64_t* b, int64_t n, int sm,
            int* status) {
  const bool unit = x->stride == 1 && y->stride == 1;
  const T al = static_cast<T>(alpha), be = static_cast<T>(beta);
  if (form == ASCB_STANDARD) {
    return unit ? launch<T, EXACT, true, true>(s, a, al, be, x, y, b, n, sm, status)
                : launch<T, EXACT, true, false>(s, a, al, be, x, y, b, n, sm, status);
  }
  return unit ? launch<T, EXACT, false, true>(s, a, al, be, x, y, b, n, sm, status)
              : launch<T, EXACT, false, false>(s, a, al, be, x, y, b, n, sm, status);
}

// bounds[2k] = first row of tile k, bounds[2k+1] = ptr[that row].
__global__ void merge_bounds_kernel(int64_t rows, const int64_t* __restrict__ ptr, int64_t items,
                                    int64_t* __restrict__ bounds, int64_t ntiles) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k > ntiles) return;
  const int64_t r = k == ntiles ? rows : first_row_at(ptr, rows, 1, k * items);
  bounds[2 * k] = r;
  bounds[2 * k + 1] = __ldg(ptr + r);
}

}  // namespace
}  // namespace ascb

extern "C" {

int64_t ascb_merge_tiles(int64_t rows, int64_t nnz) {
  if (rows <= 0) return 0;
  return (rows + nnz + ascb::kItems - 1) / ascb::kItems;
}

int ascb_merge_bounds(void* stream, const ascb_csr* a, int64_t* bounds, int64_t ntiles) {
  if (ntiles <= 0) return 0;
  const unsigned blocks = static_cast<unsigned>((ntiles + 1 + 255) / 256);
  ascb::merge_bounds_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      a->rows, a->ptr, ascb::kItems, bounds, ntiles);
  return static_cast<int>(cudaGetLastError());
}

int ascb_spmv_merge(void* stream, int dtype, int form, int exact, const ascb_csr* a,
                    double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
                    const int64_t* bounds, int64_t ntiles, int sm_count, int* status) {
  if (ntiles <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return exact ? ascb::by_form<double, true>(s, form, a, alpha, beta, x, y, bounds, ntiles, sm_count, status)
                 : ascb::by_form<double, false>(s, form, a, alpha, beta, x, y, bounds, ntiles, sm_count, status);
  }
  return exact ? ascb::by_form<float, true>(s, form, a, alpha, beta, x, y, bounds, ntiles, sm_count, status)
               : ascb::by_form<float, false>(s, form, a, alpha, beta, x, y, bounds, ntiles, sm_count, status);
}

}  // extern "C"
