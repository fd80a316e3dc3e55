// Complex (C and Z) standard SpMV and SpMM for sm_100a.
//
// Every stored entry does out += (alpha * v') * in, v' = conj(v) for the
// conjugate transpose (include/asc/sparse/blas.h:1653-1665 and 1739-1748,
// MaybeConjugate).  Arrays hold (re, im) pairs, the layout of std::complex<R>,
// aligned to R only, so components are loaded one by one.  A complex product
// (a, b)(c, d) is (ac - bd, ad + bc); in EXACT mode every product, difference
// and sum is rounded separately (the value std::complex<R> gives under GCC
// without -march for every product that is not NaN + NaN i).
//   * row products: the CSR arrays handed in are the rows of op(A) (for a
//     transposed product, the transposed structure of a plan).  One warp per
//     row, 32 products at a time; EXACT adds them to y one by one in stored
//     order, FAST sums the row with a warp tree and adds it to y once.
//   * scatter: FAST transposed products without a plan, one warp per stored
//     row, atomic adds of both components.
//   * SpMM: one thread per (row, right-hand side) in stored order, or the
//     scatter form for FAST transposed products without a plan.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;

template <typename R>
struct Cx {
  R re, im;
};

template <bool EXACT, typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  if (EXACT) {
    return {sub_rn(mul_rn(a.re, b.re), mul_rn(a.im, b.im)),
            add_rn(mul_rn(a.re, b.im), mul_rn(a.im, b.re))};
  }
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

template <bool EXACT, typename R>
__device__ __forceinline__ Cx<R> cadd(Cx<R> a, Cx<R> b) {
  if (EXACT) return {add_rn(a.re, b.re), add_rn(a.im, b.im)};
  return {a.re + b.re, a.im + b.im};
}

template <typename R>
__device__ __forceinline__ Cx<R> load(const Cx<R>* p) {
  return {__ldg(&p->re), __ldg(&p->im)};
}

template <bool CONJ, typename R>
__device__ __forceinline__ Cx<R> stored(const Cx<R>* val, int64_t q) {
  Cx<R> v = load(val + q);
  if (CONJ) v.im = -v.im;
  return v;
}

template <typename R>
__device__ __forceinline__ Cx<R> shfl(Cx<R> v, int src) {
  return {__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

template <typename R, bool EXACT, bool CONJ, bool UNIT>
__global__ void __launch_bounds__(kThreads)
complex_rows(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
             const Cx<R>* __restrict__ val, const Cx<R>* __restrict__ x, int64_t incx,
             Cx<R>* __restrict__ y, int64_t incy, Cx<R> alpha, int64_t rows) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x) >> 5; r < rows;
       r += warps) {
    const int64_t b = __ldg(ptr + r);
    const int64_t e = __ldg(ptr + r + 1);
    if (b == e) continue;  // no entry: y keeps its bits
    Cx<R>* yp = &at<UNIT>(y, r, incy);
    Cx<R> s = EXACT ? *yp : Cx<R>{R(0), R(0)};
    for (int64_t q0 = b; q0 < e; q0 += 32) {
      const int64_t q = q0 + lane;
      Cx<R> p{R(0), R(0)};
      if (q < e) {
        const Cx<R> xv = load(&at<UNIT>(x, __ldg(idx + q), incx));
        p = cmul<EXACT>(cmul<EXACT>(alpha, stored<CONJ>(val, q)), xv);
      }
      if (EXACT) {
        const int n = static_cast<int>(e - q0 < 32 ? e - q0 : 32);
        for (int k = 0; k < n; ++k) s = cadd<true>(s, shfl(p, k));
      } else {
        s = cadd<false>(s, p);
      }
    }
    if (!EXACT) {
#pragma unroll
      for (int m = 16; m > 0; m >>= 1) {
        s.re += __shfl_xor_sync(0xffffffffu, s.re, m);
        s.im += __shfl_xor_sync(0xffffffffu, s.im, m);
      }
    }
    if (lane == 0) *yp = EXACT ? s : cadd<false>(*yp, s);
  }
}

template <typename R, bool CONJ, bool UNIT>
__global__ void __launch_bounds__(kThreads)
complex_scatter(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                const Cx<R>* __restrict__ val, const Cx<R>* __restrict__ x, int64_t incx,
                Cx<R>* __restrict__ y, int64_t incy, Cx<R> alpha, int64_t rows) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x) >> 5; r < rows;
       r += warps) {
    const int64_t b = __ldg(ptr + r);
    const int64_t e = __ldg(ptr + r + 1);
    if (b == e) continue;
    const Cx<R> xr = load(&at<UNIT>(x, r, incx));
    for (int64_t q = b + lane; q < e; q += 32) {
      const Cx<R> p = cmul<false>(cmul<false>(alpha, stored<CONJ>(val, q)), xr);
      Cx<R>* yp = &at<UNIT>(y, __ldg(idx + q), incy);
      atomicAdd(&yp->re, p.re);
      atomicAdd(&yp->im, p.im);
    }
  }
}

__device__ __forceinline__ int64_t dense_at(int layout, int64_t ld, int64_t r, int64_t c) {
  return layout == ASCB_ROW_MAJOR ? r * ld + c : c * ld + r;
}

// One thread per (row of op(A), right-hand side j), j fastest.
template <typename R, bool EXACT, bool CONJ>
__global__ void __launch_bounds__(kThreads)
complex_spmm_rows(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                  const Cx<R>* __restrict__ val, const Cx<R>* __restrict__ bm, int b_layout,
                  int64_t ldb, Cx<R>* __restrict__ cm, int c_layout, int64_t ldc, int64_t k,
                  Cx<R> alpha, int64_t rows) {
  const int64_t total = rows * k;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; t < total;
       t += step) {
    const int64_t r = t / k;
    const int64_t j = t - r * k;
    const int64_t b = __ldg(ptr + r);
    const int64_t e = __ldg(ptr + r + 1);
    if (b == e) continue;
    Cx<R>* cp = cm + dense_at(c_layout, ldc, r, j);
    Cx<R> s = EXACT ? *cp : Cx<R>{R(0), R(0)};
    for (int64_t q = b; q < e; ++q) {
      const Cx<R> bv = load(bm + dense_at(b_layout, ldb, __ldg(idx + q), j));
      s = cadd<EXACT>(s, cmul<EXACT>(cmul<EXACT>(alpha, stored<CONJ>(val, q)), bv));
    }
    *cp = EXACT ? s : cadd<false>(*cp, s);
  }
}

// Transposed SpMM by scatter: one thread per (stored row r, rhs j).
template <typename R, bool CONJ>
__global__ void __launch_bounds__(kThreads)
complex_spmm_scatter(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                     const Cx<R>* __restrict__ val, const Cx<R>* __restrict__ bm, int b_layout,
                     int64_t ldb, Cx<R>* __restrict__ cm, int c_layout, int64_t ldc, int64_t k,
                     Cx<R> alpha, int64_t rows) {
  const int64_t total = rows * k;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kThreads;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x; t < total;
       t += step) {
    const int64_t r = t / k;
    const int64_t j = t - r * k;
    const Cx<R> bv = load(bm + dense_at(b_layout, ldb, r, j));
    for (int64_t q = __ldg(ptr + r); q < __ldg(ptr + r + 1); ++q) {
      const Cx<R> p = cmul<false>(cmul<false>(alpha, stored<CONJ>(val, q)), bv);
      Cx<R>* cp = cm + dense_at(c_layout, ldc, __ldg(idx + q), j);
      atomicAdd(&cp->re, p.re);
      atomicAdd(&cp->im, p.im);
    }
  }
}

unsigned Blocks(int64_t threads_needed, int sm_count) {
  const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
  int64_t b = (threads_needed + kThreads - 1) / kThreads;
  if (b > cap) b = cap;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

template <typename R, bool CONJ, bool UNIT>
int spmv_typed(cudaStream_t s, int mode, const ascb_csr* a, Cx<R> alpha, const ascb_vec* x,
               const ascb_vec* y, int sm) {
  const auto* ptr = a->ptr;
  const auto* idx = a->idx;
  const auto* val = static_cast<const Cx<R>*>(a->val);
  const auto* xd = static_cast<const Cx<R>*>(x->data);
  auto* yd = static_cast<Cx<R>*>(y->data);
  const unsigned blocks = Blocks(a->rows * 32, sm);
  if (mode == 2) {
    complex_scatter<R, CONJ, UNIT><<<blocks, kThreads, 0, s>>>(ptr, idx, val, xd, x->stride, yd,
                                                               y->stride, alpha, a->rows);
  } else if (mode == 1) {
    complex_rows<R, true, CONJ, UNIT><<<blocks, kThreads, 0, s>>>(ptr, idx, val, xd, x->stride,
                                                                  yd, y->stride, alpha, a->rows);
  } else {
    complex_rows<R, false, CONJ, UNIT><<<blocks, kThreads, 0, s>>>(ptr, idx, val, xd, x->stride,
                                                                   yd, y->stride, alpha, a->rows);
  }
  return static_cast<int>(cudaGetLastError());
}

template <typename R>
int spmv_dispatch(cudaStream_t s, int mode, int conj, const ascb_csr* a, double ar, double ai,
                  const ascb_vec* x, const ascb_vec* y, int sm) {
  const Cx<R> alpha{static_cast<R>(ar), static_cast<R>(ai)};
  const bool unit = x->stride == 1 && y->stride == 1;
  if (conj) {
    return unit ? spmv_typed<R, true, true>(s, mode, a, alpha, x, y, sm)
                : spmv_typed<R, true, false>(s, mode, a, alpha, x, y, sm);
  }
  return unit ? spmv_typed<R, false, true>(s, mode, a, alpha, x, y, sm)
              : spmv_typed<R, false, false>(s, mode, a, alpha, x, y, sm);
}

template <typename R, bool CONJ>
int spmm_typed(cudaStream_t s, int mode, const ascb_csr* a, int64_t k, const void* b,
               int b_layout, int64_t ldb, void* c, int c_layout, int64_t ldc, Cx<R> alpha,
               int sm) {
  const auto* val = static_cast<const Cx<R>*>(a->val);
  const auto* bm = static_cast<const Cx<R>*>(b);
  auto* cm = static_cast<Cx<R>*>(c);
  const unsigned blocks = Blocks(a->rows * k, sm);
  if (mode == 2) {
    complex_spmm_scatter<R, CONJ><<<blocks, kThreads, 0, s>>>(a->ptr, a->idx, val, bm, b_layout,
                                                              ldb, cm, c_layout, ldc, k, alpha,
                                                              a->rows);
  } else if (mode == 1) {
    complex_spmm_rows<R, true, CONJ><<<blocks, kThreads, 0, s>>>(
        a->ptr, a->idx, val, bm, b_layout, ldb, cm, c_layout, ldc, k, alpha, a->rows);
  } else {
    complex_spmm_rows<R, false, CONJ><<<blocks, kThreads, 0, s>>>(
        a->ptr, a->idx, val, bm, b_layout, ldb, cm, c_layout, ldc, k, alpha, a->rows);
  }
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_complex_spmv(void* stream, int dtype, int mode, int conj, const ascb_csr* a,
                                 double alpha_re, double alpha_im, const ascb_vec* x,
                                 const ascb_vec* y, int sm_count) {
  if (a->rows <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_C128) {
    return ascb::spmv_dispatch<double>(s, mode, conj, a, alpha_re, alpha_im, x, y, sm_count);
  }
  if (dtype == ASCB_C64) {
    return ascb::spmv_dispatch<float>(s, mode, conj, a, alpha_re, alpha_im, x, y, sm_count);
  }
  return static_cast<int>(cudaErrorInvalidValue);
}

extern "C" int ascb_complex_spmm(void* stream, int dtype, int mode, int conj, const ascb_csr* a,
                                 int64_t k, const void* b, int b_layout, int64_t ldb, void* c,
                                 int c_layout, int64_t ldc, double alpha_re, double alpha_im,
                                 int sm_count) {
  if (a->rows <= 0 || k <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_C128) {
    const ascb::Cx<double> al{alpha_re, alpha_im};
    return conj ? ascb::spmm_typed<double, true>(s, mode, a, k, b, b_layout, ldb, c, c_layout,
                                                 ldc, al, sm_count)
                : ascb::spmm_typed<double, false>(s, mode, a, k, b, b_layout, ldb, c, c_layout,
                                                  ldc, al, sm_count);
  }
  if (dtype == ASCB_C64) {
    const ascb::Cx<float> al{static_cast<float>(alpha_re), static_cast<float>(alpha_im)};
    return conj ? ascb::spmm_typed<float, true>(s, mode, a, k, b, b_layout, ldb, c, c_layout,
                                                ldc, al, sm_count)
                : ascb::spmm_typed<float, false>(s, mode, a, k, b, b_layout, ldb, c, c_layout,
                                                 ldc, al, sm_count);
  }
  return static_cast<int>(cudaErrorInvalidValue);
}
