// Row-ordered, bit-exact CSR SpMV for sm_100a.
//
// Reproduces the reference's serial summation order and rounding exactly:
//   compat   (src/sparse/reference_blas.cc:13-39):
//            s = +0; s = s + v_k*x_k in stored order; y = alpha*s [+ beta*y]
//   standard (include/asc/sparse/blas.h:1653-1665, ForEachStored order):
//            s = y; s = s + (alpha*v_k)*x_k in stored order; y = s
// Every product and sum uses an explicit round-to-nearest intrinsic so no FMA
// contraction can change a bit.
//
// Work decomposition (one CTA per row tile, no atomics):
//   * Tile k owns the rows whose first merge item r + ptr[r] falls in
//     [k*kItems, (k+1)*kItems); tile bounds come from row_tile_kernel.
//     All rows of a tile except the last fit in kItems nonzeros.
//   * Phase 1: the CTA streams the tile's nonzeros (values, column indices)
//     with coalesced, evict-first loads, gathers x through the read-only path
//     and writes each rounded product to shared memory -- every load in the
//     tile is in flight at once, independent of row lengths.
//   * Phase 2: one thread per row adds its products from shared memory in
//     stored order.  This is the serial dependency the reference defines; it
//     costs one shared-memory read and one add per nonzero.
//   * The last row of a tile may extend beyond the staged window (rows longer
//     than about kItems).  The whole CTA then stages the remainder in chunks
//     and thread 0 continues the same serial sum.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;
constexpr int64_t kItems = 2048;   // merge items (rows + nonzeros) per tile
constexpr int64_t kWindow = 4096;  // staged products per pass
constexpr int kBatch = 8;          // loads in flight per thread per batch
constexpr int kMaxDevices = 64;

template <typename T, bool STANDARD>
__device__ __forceinline__ T product(T alpha, T v, T xv) {
  return STANDARD ? mul_rn(mul_rn(alpha, v), xv) : mul_rn(v, xv);
}

// Stage products of nonzeros [first, first + count) into buf[0..count).
template <typename T, bool STANDARD, bool UNIT>
__device__ __forceinline__ void stage(T* __restrict__ buf, int64_t first,
                                      int64_t count,
                                      const int64_t* __restrict__ idx,
                                      const T* __restrict__ val,
                                      const T* __restrict__ x, int64_t incx,
                                      T alpha) {
  for (int64_t q0 = 0; q0 < count; q0 += int64_t{kThreads} * kBatch) {
    int64_t col[kBatch];
    T v[kBatch];
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int64_t q = q0 + j * kThreads + threadIdx.x;
      if (q < count) {
        col[j] = ld_stream(idx + first + q);
        v[j] = ld_stream(val + first + q);
      }
    }
#pragma unroll
    for (int j = 0; j < kBatch; ++j) {
      const int64_t q = q0 + j * kThreads + threadIdx.x;
      if (q < count) {
        const T xv = ld_gather(&at<UNIT>(x, col[j], incx));
        buf[q] = product<T, STANDARD>(alpha, v[j], xv);
      }
    }
  }
}

// First row r in [0, rows] with r + ptr[r] >= target (f strictly increasing).
__device__ __forceinline__ int64_t first_row_at(const int64_t* __restrict__ ptr,
                                                int64_t rows, int64_t target) {
  int64_t lo = 0;
  int64_t hi = rows;
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (mid + __ldg(ptr + mid) < target) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

template <typename T, bool STANDARD>
__device__ __forceinline__ T finish(T s, T alpha, T beta, const T* yp) {
  if (STANDARD) return s;
  T r = mul_rn(alpha, s);
  if (beta != T(0)) r = add_rn(r, mul_rn(beta, *yp));
  return r;
}

template <typename T, bool STANDARD, bool UNIT>
__global__ void __launch_bounds__(kThreads)
row_ordered_kernel(const int64_t* __restrict__ ptr,
                   const int64_t* __restrict__ idx, const T* __restrict__ val,
                   const T* __restrict__ x, int64_t incx, T* __restrict__ y,
                   int64_t incy, T alpha, T beta,
                   const int64_t* __restrict__ tile_row, int64_t rows,
                   int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  int64_t* sptr = reinterpret_cast<int64_t*>(smem);                 // kItems+1
  T* buf = reinterpret_cast<T*>(smem + (kItems + 1) * sizeof(int64_t));

  int64_t r0, r1;
  if (tile_row != nullptr) {
    r0 = tile_row[blockIdx.x];
    r1 = tile_row[blockIdx.x + 1];
  } else {
    // No partition buffer (zero-workspace calls): two threads place this
    // tile's bounds with the same search the partition kernel runs.
    __shared__ int64_t bounds[2];
    if (threadIdx.x == 0 || threadIdx.x == 32) {
      const int64_t k = blockIdx.x + (threadIdx.x == 32 ? 1 : 0);
      bounds[threadIdx.x == 32] = k >= ntiles ? rows : first_row_at(ptr, rows, k * kItems);
    }
    __syncthreads();
    r0 = bounds[0];
    r1 = bounds[1];
  }
  if (r0 == r1) return;
  const int nr = static_cast<int>(r1 - r0);  // <= kItems
  for (int i = threadIdx.x; i <= nr; i += kThreads) sptr[i] = ptr[r0 + i];
  __syncthreads();

  const int64_t base = sptr[0];
  const int64_t span = sptr[nr] - base;
  const int64_t window = span < kWindow ? span : kWindow;
  stage<T, STANDARD, UNIT>(buf, base, window, idx, val, x, incx, alpha);
  __syncthreads();

  // Phase 2: one thread per row, serial sum in stored order.
  for (int i = threadIdx.x; i < nr; i += kThreads) {
    const int64_t b = sptr[i] - base;
    const int64_t e = sptr[i + 1] - base;
    if (e > window) continue;  // only the tile's last row; handled below
    T* yp = &at<UNIT>(y, r0 + i, incy);
    T s = STANDARD ? *yp : T(0);
    for (int64_t q = b; q < e; ++q) s = add_rn(s, buf[q]);
    *yp = finish<T, STANDARD>(s, alpha, beta, yp);
  }
  if (span <= kWindow) return;  // uniform across the CTA

  // Long last row: continue the serial sum over staged chunks.
  __shared__ T carry;
  const int64_t b_last = sptr[nr - 1] - base;
  T* y_last = &at<UNIT>(y, r1 - 1, incy);
  if (threadIdx.x == 0) {
    T s = STANDARD ? *y_last : T(0);
    for (int64_t q = b_last; q < window; ++q) s = add_rn(s, buf[q]);
    carry = s;
  }
  for (int64_t done = window; done < span; done += kWindow) {
    __syncthreads();  // thread 0 finished reading buf
    const int64_t count = span - done < kWindow ? span - done : kWindow;
    stage<T, STANDARD, UNIT>(buf, base + done, count, idx, val, x, incx, alpha);
    __syncthreads();
    if (threadIdx.x == 0) {
      T s = carry;
      for (int64_t q = 0; q < count; ++q) s = add_rn(s, buf[q]);
      carry = s;
    }
  }
  if (threadIdx.x == 0) *y_last = finish<T, STANDARD>(carry, alpha, beta, y_last);
}

template <typename T>
constexpr size_t smem_bytes() {
  return (kItems + 1) * sizeof(int64_t) + kWindow * sizeof(T);
}

template <typename T, bool STANDARD, bool UNIT>
int launch(cudaStream_t stream, const ascb_csr* a, T alpha, T beta,
           const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
           int64_t ntiles) {
  auto kernel = row_ordered_kernel<T, STANDARD, UNIT>;
  // The shared-memory opt-in is a per-device function attribute.
  static bool configured[kMaxDevices] = {};
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (device < 0 || device >= kMaxDevices || !configured[device]) {
    e = cudaFuncSetAttribute(kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem_bytes<T>()));
    if (e != cudaSuccess) return static_cast<int>(e);
    if (device >= 0 && device < kMaxDevices) configured[device] = true;
  }
  kernel<<<static_cast<unsigned>(ntiles), kThreads, smem_bytes<T>(), stream>>>(
      a->ptr, a->idx, static_cast<const T*>(a->val),
      static_cast<const T*>(x->data), x->stride, static_cast<T*>(y->data),
      y->stride, alpha, beta, tile_row, a->rows, ntiles);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int dispatch(cudaStream_t s, int form, const ascb_csr* a, double alpha,
             double beta, const ascb_vec* x, const ascb_vec* y,
             const int64_t* tile_row, int64_t ntiles) {
  const bool unit = x->stride == 1 && y->stride == 1;
  const T al = static_cast<T>(alpha);
  const T be = static_cast<T>(beta);
  if (form == ASCB_STANDARD) {
    return unit ? launch<T, true, true>(s, a, al, be, x, y, tile_row, ntiles)
                : launch<T, true, false>(s, a, al, be, x, y, tile_row, ntiles);
  }
  return unit ? launch<T, false, true>(s, a, al, be, x, y, tile_row, ntiles)
              : launch<T, false, false>(s, a, al, be, x, y, tile_row, ntiles);
}

}  // namespace
}  // namespace ascb

extern "C" {

int64_t ascb_row_ordered_items(int /*dtype*/) { return ascb::kItems; }

int ascb_spmv_row_ordered(void* stream, int dtype, int form, const ascb_csr* a,
                          double alpha, double beta, const ascb_vec* x,
                          const ascb_vec* y, const int64_t* tile_row,
                          int64_t ntiles) {
  if (ntiles <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == ASCB_F64
             ? ascb::dispatch<double>(s, form, a, alpha, beta, x, y, tile_row,
                                      ntiles)
             : ascb::dispatch<float>(s, form, a, alpha, beta, x, y, tile_row,
                                     ntiles);
}

}  // extern "C"
