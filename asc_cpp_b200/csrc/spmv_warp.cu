// Warp-tiled, software-pipelined CSR SpMV for sm_100a (the default SpMV).
//
// Each warp works through a contiguous range of small row tiles on its own --
// no CTA-wide barriers -- so an SM keeps dozens of tiles, and thousands of
// independent x gathers, in flight.  That is what power-law matrices need: the
// streamed bytes (values and int64 column indices) are only part of the memory
// work; the rest is dependent random reads of x, which hit L2.
//
// Tiles.  With weight W = kItems / 32, tile t owns the rows r whose weighted
// start W*r + ptr[r] falls in [t*kItems, (t+1)*kItems) (row_tile_kernel with
// weight W).  A tile therefore has at most 32 rows -- one per lane -- and all of
// its rows except the last hold fewer than kItems nonzeros.
//
// Pipeline.  A tile costs three dependent memory round trips: row bounds
// (ptr) -> column indices -> x gathers.  Step t of a warp overlaps them across
// three consecutive tiles:
//     cp.async  ptr of tile t+2              -> shared slot (t+2) % 3
//     cp.async  column indices of tile t+1   -> shared ring (t+1) % 2
//     gather x for tile t (values streamed evict-first), form the products in
//     shared memory, one lane per row sums its products in stored order, y.
// A row longer than the staged window (kItems nonzeros) is finished by the
// whole warp in further windows: in EXACT mode its owner lane keeps the serial
// sum, in FAST mode the lanes reduce each window with a butterfly.
//
// EXACT mode reproduces the reference's rounding bit for bit:
//   compat   (src/sparse/reference_blas.cc:13-39): s = +0; s = s + v*x ...;
//            y = alpha*s (+ beta*y)
//   standard (include/asc/sparse/blas.h:1653-1665): s = y; s = s + (alpha*v)*x
// FAST mode differs only in the reduction order of long rows; its error is
// within gamma_{n+2}(|alpha||A||x| + |beta||y|).
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kThreads = kWarpsPerCta * 32;
constexpr int64_t kItems = 256;        // weighted items per tile
constexpr int64_t kRowWeight = kItems / 32;
constexpr int kPerLane = kItems / 32;  // staged products per lane
constexpr int kChunk = 32;             // tile bounds cached per warp
#ifndef ASCB_WARP_BATCH
#define ASCB_WARP_BATCH 4
#endif
constexpr int kBatch = ASCB_WARP_BATCH;  // gathers in flight per lane per batch
#ifndef ASCB_WARP_MIN_CTAS
#define ASCB_WARP_MIN_CTAS 6
#endif
constexpr int kMinCtasPerSm = ASCB_WARP_MIN_CTAS;  // resident CTAs per SM (register budget)
constexpr int kMaxDevices = 64;

template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T product(T alpha, T v, T xv) {
  if (STANDARD) return mul_rn(mul_rn(alpha, v), xv);
  return EXACT ? mul_rn(v, xv) : v * xv;
}

template <bool EXACT, typename T>
__device__ __forceinline__ T add(T a, T b) {
  return EXACT ? add_rn(a, b) : a + b;
}

template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T finish(T s, T alpha, T beta, const T* yp) {
  if (STANDARD) return s;
  if (EXACT) {
    T r = mul_rn(alpha, s);
    if (beta != T(0)) r = add_rn(r, mul_rn(beta, *yp));
    return r;
  }
  return beta != T(0) ? fma(alpha, s, beta * *yp) : alpha * s;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Product q lives at padded slot pq(q) = q + q/16.  Rows summed one per lane
// start at arbitrary offsets; with rows of 16 products the unpadded layout
// put all 16 lanes of a half-warp on one bank.  The pad skews them apart,
// while the staging writes (32 consecutive q) stay conflict-free.
__device__ __forceinline__ int pq(int q) { return q + (q >> 4); }

// Per-warp shared state.
template <typename T>
struct WarpSmem {
  int64_t ring[2][kItems];           // column indices, double buffered
  int64_t rows[3][kChunk + 1];       // ptr[r0 .. r0 + nr] per pipelined tile
  int64_t bnd[kChunk + 1];           // first row of tiles c0 .. c0 + kChunk
  T prod[kItems + kItems / 16];      // products, padded layout
};

template <typename T>
__device__ __forceinline__ T* products(WarpSmem<T>& w, int /*slot*/) {
  return w.prod;
}

// Stage the products of nonzeros [first, first + count), count <= kItems,
// into buf with plain loads (used for the continuation windows of long rows).
template <bool EXACT, bool STANDARD, bool UNIT, typename T>
__device__ __forceinline__ void stage(T* __restrict__ buf, int lane, int64_t first, int count,
                                      const int64_t* __restrict__ idx, const T* __restrict__ val,
                                      const T* __restrict__ x, int64_t incx, T alpha) {
#pragma unroll 1
  for (int j0 = 0; j0 < kPerLane; j0 += kBatch) {
    if (j0 * 32 >= count) break;
    int64_t col[kBatch];
    T v[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int q = (j0 + j) * 32 + lane;
      if (q < count) {
        col[j] = ld_stream(idx + first + q);
        v[j] = ld_stream(val + first + q);
      }
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int q = (j0 + j) * 32 + lane;
      if (q < count) {
        buf[pq(q)] = product<EXACT, STANDARD>(alpha, v[j], ld_gather(&at<UNIT>(x, col[j], incx)));
      }
    }
  }
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT>
__global__ void __launch_bounds__(kThreads, kMinCtasPerSm)
warp_tile_kernel(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                 const T* __restrict__ val, const T* __restrict__ x, int64_t incx,
                 T* __restrict__ y, int64_t incy, T alpha, T beta,
                 const int64_t* __restrict__ tile_row, int64_t ntiles, int64_t rows) {
  __shared__ WarpSmem<T> smem_all[kWarpsPerCta];
  const int lane = threadIdx.x & 31;
  WarpSmem<T>& w = smem_all[threadIdx.x >> 5];

  const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + (threadIdx.x >> 5);
  const int64_t warp_count = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  const int64_t per_warp = (ntiles + warp_count - 1) / warp_count;
  const int64_t tb = warp_id * per_warp;
  const int64_t te = tb + per_warp < ntiles ? tb + per_warp : ntiles;
  if (tb >= te) return;

  // Tile bounds, kChunk tiles at a time.  Without a partition buffer the
  // lanes place the bounds by the partition kernel's binary search.
  int64_t c0 = -2 * kChunk;
  auto tile_bounds = [&](int64_t u, int64_t& r0, int& nr) {
    if (u + 1 > c0 + kChunk) {
      __syncwarp();
      c0 = u;
      for (int i = lane; i <= kChunk; i += 32) {
        const int64_t v = c0 + i;
        int64_t b = rows;
        if (v < ntiles) {
          b = tile_row != nullptr ? __ldg(tile_row + v)
                                  : first_row_at(ptr, rows, kRowWeight, v * kItems);
        }
        w.bnd[i] = b;
      }
      __syncwarp();
    }
    r0 = w.bnd[u - c0];
    nr = static_cast<int>(w.bnd[u - c0 + 1] - r0);
  };
  // Stage P: copy ptr[r0 .. r0 + nr] of tile u into rows slot k.
  auto copy_rows = [&](int64_t u, int k, int64_t& r0, int& nr) {
    r0 = 0;
    nr = 0;
    if (u >= te) return;
    tile_bounds(u, r0, nr);
    if (lane <= nr) cp_async8(&w.rows[k][lane], ptr + r0 + lane);
    if (lane == 0 && nr == 32) cp_async8(&w.rows[k][32], ptr + r0 + 32);
  };
  // Stage I: copy the first window of column indices of the tile in rows
  // slot k (its ptr values have landed) into ring slot s.
  auto copy_indices = [&](int k, int nr, int s) {
    if (nr == 0) return;
    const int64_t base = w.rows[k][0];
    const int64_t span = w.rows[k][nr] - base;
    const int count = static_cast<int>(span < kItems ? span : kItems);
    for (int q = lane; q < count; q += 32) cp_async8(&w.ring[s][q], idx + base + q);
  };

  int64_t r0_cur, r0_next, r0_after;
  int nr_cur, nr_next, nr_after;
  copy_rows(tb, 0, r0_cur, nr_cur);
  copy_rows(tb + 1, 1, r0_next, nr_next);
  cp_async_commit();
  cp_async_wait_all();
  __syncwarp();
  copy_indices(0, nr_cur, 0);
  cp_async_commit();

  for (int64_t t = tb; t < te; ++t) {
    const int step = static_cast<int>(t - tb);
    const int k_cur = step % 3;
    const int s_cur = step & 1;
    cp_async_wait_all();  // rows of t+1 and indices of t have landed
    __syncwarp();
    copy_rows(t + 2, (step + 2) % 3, r0_after, nr_after);
    copy_indices((step + 1) % 3, nr_next, s_cur ^ 1);
    cp_async_commit();

    if (nr_cur > 0) {
      const int nr = nr_cur;
      const int64_t base = w.rows[k_cur][0];
      const int64_t span = w.rows[k_cur][nr] - base;
      const int count = static_cast<int>(span < kItems ? span : kItems);
      T* buf = products(w, s_cur);
      // gather x and form the products of the first window
#pragma unroll 1
      for (int j0 = 0; j0 < kPerLane; j0 += kBatch) {
        if (j0 * 32 >= count) break;
        int64_t col[kBatch];
        T v[kBatch];
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
          const int q = (j0 + j) * 32 + lane;
          if (q < count) {
            col[j] = w.ring[s_cur][q];
            v[j] = ld_stream(val + base + q);
          }
        }
#pragma unroll
        for (int j = 0; j < kBatch; ++j) {
          const int q = (j0 + j) * 32 + lane;
          if (q < count) {
            buf[pq(q)] = product<EXACT, STANDARD>(alpha, v[j], ld_gather(&at<UNIT>(x, col[j], incx)));
          }
        }
      }
      __syncwarp();
      const int owner = nr - 1;  // the only row that may outrun the window
      T* yp = lane < nr ? &at<UNIT>(y, r0_cur + lane, incy) : nullptr;
      T s = T(0);
      if (lane < nr) {
        const int64_t rb = w.rows[k_cur][lane] - base;
        const int64_t re = w.rows[k_cur][lane + 1] - base;
        s = STANDARD ? *yp : T(0);
        const int e = re < count ? static_cast<int>(re) : count;
        for (int q = static_cast<int>(rb); q < e; ++q) s = add<EXACT>(s, buf[pq(q)]);
        if (re <= count) *yp = finish<EXACT, STANDARD>(s, alpha, beta, yp);
      }
      if (span > kItems) {
        // the last row continues: further windows, loaded synchronously
        for (int64_t done = kItems; done < span; done += kItems) {
          __syncwarp();
          const int n = static_cast<int>(span - done < kItems ? span - done : kItems);
          stage<EXACT, STANDARD, UNIT>(buf, lane, base + done, n, idx, val, x, incx, alpha);
          __syncwarp();
          if (EXACT) {
            if (lane == owner) {
              for (int q = 0; q < n; ++q) s = add_rn(s, buf[pq(q)]);
            }
          } else {
            T part = T(0);
            for (int q = lane; q < n; q += 32) part += buf[pq(q)];
#pragma unroll
            for (int m = 16; m > 0; m >>= 1) part += shfl_xor(part, m);
            if (lane == owner) s += part;
          }
        }
        if (lane == owner) *yp = finish<EXACT, STANDARD>(s, alpha, beta, yp);
      }
    }
    __syncwarp();  // ring slot and products are free for reuse
    r0_cur = r0_next;
    nr_cur = nr_next;
    r0_next = r0_after;
    nr_next = nr_after;
  }
  cp_async_wait_all();
}

// CTAs that fit on one SM at once (queried once per device and instantiation):
// the grid is exactly one resident wave, so the static split of tiles over
// warps is balanced.
template <typename T, bool EXACT, bool STANDARD, bool UNIT, typename Kernel>
int resident_ctas_per_sm(Kernel kernel) {
  static int cached[kMaxDevices] = {};  // one cache per instantiation
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return 1;
  if (cached[device] == 0) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, 0) != cudaSuccess ||
        n <= 0) {
      (void)cudaGetLastError();
      n = 1;
    }
    cached[device] = n;
  }
  return cached[device];
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT>
int launch(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
           const ascb_vec* y, const int64_t* tile_row, int64_t ntiles, int sm_count) {
  auto kernel = warp_tile_kernel<T, EXACT, STANDARD, UNIT>;
  // at least ~4 tiles per warp so the pipeline fills
  const int64_t warps_needed = (ntiles + 3) / 4;
  const int64_t ctas_needed = (warps_needed + kWarpsPerCta - 1) / kWarpsPerCta;
  const int64_t resident =
      static_cast<int64_t>(sm_count > 0 ? sm_count : 148) *
      resident_ctas_per_sm<T, EXACT, STANDARD, UNIT>(kernel);
  const unsigned blocks = static_cast<unsigned>(
      ctas_needed < 1 ? 1 : (ctas_needed < resident ? ctas_needed : resident));
  kernel<<<blocks, kThreads, 0, stream>>>(
      a->ptr, a->idx, static_cast<const T*>(a->val), static_cast<const T*>(x->data), x->stride,
      static_cast<T*>(y->data), y->stride, alpha, beta, tile_row, ntiles, a->rows);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, bool EXACT>
int by_form(cudaStream_t s, int form, const ascb_csr* a, double alpha, double beta,
            const ascb_vec* x, const ascb_vec* y, const int64_t* tiles, int64_t n, int sm) {
  const bool unit = x->stride == 1 && y->stride == 1;
  const T al = static_cast<T>(alpha), be = static_cast<T>(beta);
  if (form == ASCB_STANDARD) {
    return unit ? launch<T, EXACT, true, true>(s, a, al, be, x, y, tiles, n, sm)
                : launch<T, EXACT, true, false>(s, a, al, be, x, y, tiles, n, sm);
  }
  return unit ? launch<T, EXACT, false, true>(s, a, al, be, x, y, tiles, n, sm)
              : launch<T, EXACT, false, false>(s, a, al, be, x, y, tiles, n, sm);
}

}  // namespace
}  // namespace ascb

extern "C" {

int64_t ascb_warp_tile_items(void) { return ascb::kItems; }
int64_t ascb_warp_tile_row_weight(void) { return ascb::kRowWeight; }

int ascb_spmv_warp(void* stream, int dtype, int form, int exact, const ascb_csr* a,
                   double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
                   const int64_t* tile_row, int64_t ntiles, int sm_count) {
  if (ntiles <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return exact ? ascb::by_form<double, true>(s, form, a, alpha, beta, x, y, tile_row, ntiles, sm_count)
                 : ascb::by_form<double, false>(s, form, a, alpha, beta, x, y, tile_row, ntiles, sm_count);
  }
  return exact ? ascb::by_form<float, true>(s, form, a, alpha, beta, x, y, tile_row, ntiles, sm_count)
               : ascb::by_form<float, false>(s, form, a, alpha, beta, x, y, tile_row, ntiles, sm_count);
}

}  // extern "C"
