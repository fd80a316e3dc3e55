// Vector-CSR SpMV for sm_100a: a group of LANES threads (1..32) owns a row,
// strides through its nonzeros with fused multiply-adds and combines the lane
// partials with a butterfly of warp shuffles.  Persistent grid-stride CTAs
// (a whole number of waves over the 148 SMs).  Numerics: each lane's partial is
// a contracted running sum and the butterfly reorders it, so results satisfy
// |y - y_ref| <= gamma_{n+2} (|alpha||A||x| + |beta||y|) rather than being
// bit-identical to the serial order.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;
constexpr int kUnroll = 4;

template <typename T, int LANES, bool STANDARD, bool UNIT>
__global__ void __launch_bounds__(kThreads)
vector_kernel(int64_t rows, const int64_t* __restrict__ ptr,
              const int64_t* __restrict__ idx, const T* __restrict__ val,
              const T* __restrict__ x, int64_t incx, T* __restrict__ y,
              int64_t incy, T alpha, T beta) {
  constexpr int kGroups = kThreads / LANES;
  const int lane = threadIdx.x % LANES;
  const int64_t first =
      static_cast<int64_t>(blockIdx.x) * kGroups + threadIdx.x / LANES;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kGroups;
  for (int64_t row = first; row < rows; row += step) {
    const int64_t b = __ldg(ptr + row);
    const int64_t e = __ldg(ptr + row + 1);
    T acc[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) acc[u] = T(0);
    int64_t q = b + lane;
    for (; q + (kUnroll - 1) * LANES < e; q += kUnroll * LANES) {
      int64_t col[kUnroll];
      T v[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        col[u] = ld_stream(idx + q + u * LANES);
        v[u] = ld_stream(val + q + u * LANES);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        acc[u] = fma(v[u], ld_gather(&at<UNIT>(x, col[u], incx)), acc[u]);
      }
    }
    for (; q < e; q += LANES) {
      acc[0] = fma(ld_stream(val + q),
                   ld_gather(&at<UNIT>(x, ld_stream(idx + q), incx)), acc[0]);
    }
    T s = (acc[0] + acc[1]) + (acc[2] + acc[3]);
#pragma unroll
    for (int m = LANES / 2; m > 0; m >>= 1) s += shfl_xor(s, m, LANES);
    if (lane == 0) {
      T* yp = &at<UNIT>(y, row, incy);
      if (STANDARD) {
        *yp = fma(alpha, s, *yp);
      } else {
        *yp = beta != T(0) ? fma(alpha, s, beta * *yp) : alpha * s;
      }
    }
  }
}

template <typename T, int LANES, bool STANDARD, bool UNIT>
int launch(cudaStream_t stream, const ascb_csr* a, T alpha, T beta,
           const ascb_vec* x, const ascb_vec* y, int sm_count) {
  constexpr int kGroups = kThreads / LANES;
  const int64_t needed = (a->rows + kGroups - 1) / kGroups;
  const int64_t resident = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
  const unsigned blocks =
      static_cast<unsigned>(needed < resident ? needed : resident);
  vector_kernel<T, LANES, STANDARD, UNIT><<<blocks, kThreads, 0, stream>>>(
      a->rows, a->ptr, a->idx, static_cast<const T*>(a->val),
      static_cast<const T*>(x->data), x->stride, static_cast<T*>(y->data),
      y->stride, alpha, beta);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, int LANES>
int by_form(cudaStream_t s, int form, const ascb_csr* a, T al, T be,
            const ascb_vec* x, const ascb_vec* y, int sm) {
  const bool unit = x->stride == 1 && y->stride == 1;
  if (form == ASCB_STANDARD) {
    return unit ? launch<T, LANES, true, true>(s, a, al, be, x, y, sm)
                : launch<T, LANES, true, false>(s, a, al, be, x, y, sm);
  }
  return unit ? launch<T, LANES, false, true>(s, a, al, be, x, y, sm)
              : launch<T, LANES, false, false>(s, a, al, be, x, y, sm);
}

template <typename T>
int by_lanes(cudaStream_t s, int form, int lanes, const ascb_csr* a,
             double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
             int sm) {
  const T al = static_cast<T>(alpha);
  const T be = static_cast<T>(beta);
  switch (lanes) {
    case 1: return by_form<T, 1>(s, form, a, al, be, x, y, sm);
    case 2: return by_form<T, 2>(s, form, a, al, be, x, y, sm);
    case 4: return by_form<T, 4>(s, form, a, al, be, x, y, sm);
    case 8: return by_form<T, 8>(s, form, a, al, be, x, y, sm);
    case 16: return by_form<T, 16>(s, form, a, al, be, x, y, sm);
    case 32: return by_form<T, 32>(s, form, a, al, be, x, y, sm);
    default: return static_cast<int>(cudaErrorInvalidValue);
  }
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_spmv_vector(void* stream, int dtype, int form, int lanes,
                                const ascb_csr* a, double alpha, double beta,
                                const ascb_vec* x, const ascb_vec* y,
                                int sm_count) {
  if (a->rows <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == ASCB_F64
             ? ascb::by_lanes<double>(s, form, lanes, a, alpha, beta, x, y,
                                      sm_count)
             : ascb::by_lanes<float>(s, form, lanes, a, alpha, beta, x, y,
                                     sm_count);
}
