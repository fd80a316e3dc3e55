// Level-1 sparse BLAS on an indexed vector (indices sorted and unique, the
// reference's canonical indexed storage) for sm_100a:
//   dot        r = sum_k v'_k x[i_k]        (v' = conj(v) when conjugated)
//   axpy       x[i_k] += alpha v_k
//   gather     v_k = x[i_k]
//   gather0    v_k = x[i_k]; x[i_k] = 0
//   scatter    x[i_k] = v_k
// (include/asc/sparse/blas.h:1340-1600; the CUDA facet's StandardLevel1Kernel,
// src/sparse/cuda/kernels.cu:200-258, runs the dot on one thread).
// The element-wise operations touch distinct x entries, so they run one
// thread per entry and are exact (axpy rounds alpha v and the sum separately,
// as the reference does).  The dot in DETERMINISTIC mode keeps the
// reference's serial order and rounding: one warp forms 32 products at a time
// and lane 0 adds them in stored order; otherwise a grid reduction with a
// fixed tree (reproducible run to run) writes the sum.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

template <typename R>
struct Cx {
  R re, im;
};

template <typename T>
struct Ops {  // real
  using S = T;
  __device__ static T zero() { return T(0); }
  __device__ static T mul(T a, T b, bool exact) { return exact ? mul_rn(a, b) : a * b; }
  __device__ static T add(T a, T b, bool exact) { return exact ? add_rn(a, b) : a + b; }
  __device__ static T conj(T a) { return a; }
  __device__ static T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
  __device__ static T shfl_down(T v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
};

template <typename R>
struct Ops<Cx<R>> {
  using T = Cx<R>;
  __device__ static T zero() { return {R(0), R(0)}; }
  __device__ static T mul(T a, T b, bool exact) {
    if (exact) {
      return {sub_rn(mul_rn(a.re, b.re), mul_rn(a.im, b.im)),
              add_rn(mul_rn(a.re, b.im), mul_rn(a.im, b.re))};
    }
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  }
  __device__ static T add(T a, T b, bool exact) {
    return exact ? T{add_rn(a.re, b.re), add_rn(a.im, b.im)} : T{a.re + b.re, a.im + b.im};
  }
  __device__ static T conj(T a) { return {a.re, -a.im}; }
  __device__ static T shfl(T v, int src) {
    return {__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
  }
  __device__ static T shfl_down(T v, int d) {
    return {__shfl_down_sync(0xffffffffu, v.re, d), __shfl_down_sync(0xffffffffu, v.im, d)};
  }
};

template <typename T>
__device__ __forceinline__ T& dense_at(T* x, int64_t i, int64_t inc) {
  return x[i * inc];
}

template <typename T>
__global__ void level1_elementwise(int op, const int64_t* __restrict__ idx, T* val, int64_t n,
                                   T* x, int64_t incx, T alpha) {
  using O = Ops<T>;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < n;
       q += step) {
    T& xi = dense_at(x, __ldg(idx + q), incx);
    switch (op) {
      case ASCB_L1_AXPY:
        xi = O::add(xi, O::mul(alpha, val[q], true), true);
        break;
      case ASCB_L1_GATHER:
        val[q] = xi;
        break;
      case ASCB_L1_GATHER_ZERO:
        val[q] = xi;
        xi = O::zero();
        break;
      case ASCB_L1_SCATTER:
        xi = val[q];
        break;
      default:
        break;
    }
  }
}

// Dot in stored order (one warp): 32 products at a time, added by lane 0.
template <typename T, bool CONJ>
__global__ void level1_dot_ordered(const int64_t* __restrict__ idx, const T* __restrict__ val,
                                   int64_t n, const T* __restrict__ x, int64_t incx, T* result) {
  using O = Ops<T>;
  const int lane = threadIdx.x & 31;
  T sum = O::zero();
  for (int64_t q0 = 0; q0 < n; q0 += 32) {
    const int64_t q = q0 + lane;
    T p = O::zero();
    if (q < n) {
      const T v = CONJ ? O::conj(val[q]) : val[q];
      p = O::mul(v, dense_at(x, __ldg(idx + q), incx), true);
    }
    const int m = static_cast<int>(n - q0 < 32 ? n - q0 : 32);
    for (int k = 0; k < m; ++k) {
      const T pk = O::shfl(p, k);
      if (lane == 0) sum = O::add(sum, pk, true);
    }
  }
  if (lane == 0) *result = sum;
}

constexpr int kDotThreads = 256;

// Contracted dot, pass 1: each block reduces a contiguous range (fixed tree).
template <typename T, bool CONJ>
__global__ void level1_dot_partial(const int64_t* __restrict__ idx, const T* __restrict__ val,
                                   int64_t n, const T* __restrict__ x, int64_t incx,
                                   T* __restrict__ partial) {
  using O = Ops<T>;
  __shared__ T warp_sums[kDotThreads / 32];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  T acc = O::zero();
  for (int64_t q = b + threadIdx.x; q < e; q += kDotThreads) {
    const T v = CONJ ? O::conj(val[q]) : val[q];
    acc = O::add(acc, O::mul(v, dense_at(x, __ldg(idx + q), incx), false), false);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) acc = O::add(acc, O::shfl_down(acc, d), false);
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    T s = O::zero();
    for (int w = 0; w < kDotThreads / 32; ++w) s = O::add(s, warp_sums[w], false);
    partial[blockIdx.x] = s;
  }
}

// Pass 2: one thread adds the block sums in order.
template <typename T>
__global__ void level1_dot_final(const T* __restrict__ partial, int count, T* result) {
  using O = Ops<T>;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  T s = O::zero();
  for (int i = 0; i < count; ++i) s = O::add(s, partial[i], false);
  *result = s;
}

template <typename T>
int run(cudaStream_t s, int op, int conj, int exact, const int64_t* idx, void* val, int64_t n,
        void* x, int64_t incx, void* result, T alpha, void* scratch, int sm) {
  T* v = static_cast<T*>(val);
  T* xd = static_cast<T*>(x);
  if (op == ASCB_L1_DOT) {
    T* r = static_cast<T*>(result);
    if (exact || n < 4096 || scratch == nullptr) {
      if (conj) {
        level1_dot_ordered<T, true><<<1, 32, 0, s>>>(idx, v, n, xd, incx, r);
      } else {
        level1_dot_ordered<T, false><<<1, 32, 0, s>>>(idx, v, n, xd, incx, r);
      }
    } else {
      const int blocks = ASCB_L1_DOT_BLOCKS;
      T* partial = static_cast<T*>(scratch);
      if (conj) {
        level1_dot_partial<T, true><<<blocks, kDotThreads, 0, s>>>(idx, v, n, xd, incx, partial);
      } else {
        level1_dot_partial<T, false><<<blocks, kDotThreads, 0, s>>>(idx, v, n, xd, incx, partial);
      }
      level1_dot_final<T><<<1, 32, 0, s>>>(partial, blocks, r);
    }
    return static_cast<int>(cudaGetLastError());
  }
  if (n <= 0) return 0;
  int64_t blocks = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * 8;
  if (blocks > cap) blocks = cap;
  level1_elementwise<T><<<static_cast<unsigned>(blocks), 256, 0, s>>>(op, idx, v, n, xd, incx,
                                                                      alpha);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_level1(void* stream, int dtype, int op, int conj, int exact,
                           const int64_t* idx, void* val, int64_t n, void* x, int64_t incx,
                           void* result, double alpha_re, double alpha_im, void* scratch,
                           int sm_count) {
  using namespace ascb;
  auto s = static_cast<cudaStream_t>(stream);
  switch (dtype) {
    case ASCB_F64:
      return run<double>(s, op, conj, exact, idx, val, n, x, incx, result, alpha_re, scratch,
                         sm_count);
    case ASCB_F32:
      return run<float>(s, op, conj, exact, idx, val, n, x, incx, result,
                        static_cast<float>(alpha_re), scratch, sm_count);
    case ASCB_C128:
      return run<Cx<double>>(s, op, conj, exact, idx, val, n, x, incx, result,
                             Cx<double>{alpha_re, alpha_im}, scratch, sm_count);
    case ASCB_C64:
      return run<Cx<float>>(s, op, conj, exact, idx, val, n, x, incx, result,
                            Cx<float>{static_cast<float>(alpha_re), static_cast<float>(alpha_im)},
                            scratch, sm_count);
    default:
      return static_cast<int>(cudaErrorInvalidValue);
  }
}
