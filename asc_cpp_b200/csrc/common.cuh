// Device-side helpers shared by the sm_100a Sparse BLAS kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ascb {

// Round-to-nearest arithmetic that the compiler may not contract into an FMA.
// The reference's x86-64 build rounds every * and + separately
// (src/sparse/reference_blas.cc:32-37 compiled without -march), so the
// bit-exact kernels use these exclusively.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// Streamed, read-once operands (values, column indices): evict-first so the
// gathered x vector keeps its place in L2.
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ int64_t ld_stream(const int64_t* p) {
  return static_cast<int64_t>(__ldcs(reinterpret_cast<const long long*>(p)));
}

// 32-byte streamed loads (sm_100: one request per lane for 4 int64 / 4
// double / 8 float); the address must be 32-byte aligned.
__device__ __forceinline__ void ld_stream32(const int64_t* p, int64_t* o) {
  asm volatile("ld.global.cs.v4.s64 {%0, %1, %2, %3}, [%4];"
               : "=l"(o[0]), "=l"(o[1]), "=l"(o[2]), "=l"(o[3]) : "l"(p));
}
__device__ __forceinline__ void ld_stream32(const double* p, double* o) {
  asm volatile("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3]) : "l"(p));
}
__device__ __forceinline__ void ld_stream32(const float* p, float* o) {
  asm volatile("ld.global.cs.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]), "=f"(o[4]), "=f"(o[5]),
                 "=f"(o[6]), "=f"(o[7])
               : "l"(p));
}

// Gathered operand (x): read-only path, cached in L1 and L2.
#ifndef ASCB_GATHER_NOALLOC
template <typename T>
__device__ __forceinline__ T ld_gather(const T* p) { return __ldg(p); }
#else
// variant: no L1 allocation for the gathers
__device__ __forceinline__ double ld_gather(const double* p) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_gather(const float* p) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
#endif

// Strided element access; `stride` may be negative (pointer = logical 0).
template <bool UNIT, typename T>
__device__ __forceinline__ T& at(T* base, int64_t i, int64_t stride) {
  return UNIT ? base[i] : base[i * stride];
}
template <bool UNIT, typename T>
__device__ __forceinline__ const T& at(const T* base, int64_t i, int64_t stride) {
  return UNIT ? base[i] : base[i * stride];
}

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int mask, int width = 32) {
  return __shfl_xor_sync(0xffffffffu, v, mask, width);
}

// First row r in [0, rows] with weight*r + ptr[r] >= target.  The key is
// strictly increasing in r, so row tiles defined by it are contiguous, and a
// tile spanning `items` keys holds at most items/weight rows.
__device__ __forceinline__ int64_t first_row_at(const int64_t* __restrict__ ptr, int64_t rows,
                                                int64_t weight, int64_t target) {
  int64_t lo = 0;
  int64_t hi = rows;
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (weight * mid + __ldg(ptr + mid) < target) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

}  // namespace ascb
