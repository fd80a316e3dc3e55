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

// ---- TMA bulk copies into this CTA's shared memory, and mbarriers ---------
// (plain 1-D cp.async.bulk global -> shared, completing on an mbarrier; no
// cluster multicast anywhere)
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n .reg .b64 st;\n"
      " mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}
// try_wait with a suspend-time hint: the warp sleeps in hardware (up to the
// hint, in ns) instead of re-issuing the poll.
// suspend_ns = 0: no hint (the hardware's own time limit).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity,
                                              uint32_t suspend_ns) {
  uint32_t ok;
  if (suspend_ns == 0) {
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
  } else {
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(suspend_ns)
        : "memory");
  }
  return ok != 0;
}
// Suspend hint of the pipelined kernels' stage waits (0, 200 and 2000 ns
// measured the same on B200: the waiting warp resumes when the phase
// completes).
constexpr uint32_t kTmaSuspendNs = 2000;
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// A bulk copy of elements [first, first + count) of an array of `total`
// elements of size E: the 16-byte aligned part goes through TMA into
// dst + (first - aligned first); `tail` elements at the very end of the array
// that a 16-byte rounded copy would overrun are fetched by plain loads.
template <int E>
struct CopyPlan {
  int64_t g0;        // first element copied by TMA (16-byte aligned)
  uint32_t bytes;    // TMA bytes (multiple of 16, may be 0)
  int lead;          // smem slot of element `first`
  int64_t tail0;     // first element loaded by plain loads
  int tail;          // number of such elements
};

template <int E>
__device__ __forceinline__ CopyPlan<E> plan_copy(int64_t first, int64_t count, int64_t total) {
  constexpr int64_t kPer16 = 16 / E;
  CopyPlan<E> c;
  if (count <= 0) {
    c.g0 = first;
    c.bytes = 0;
    c.lead = 0;
    c.tail0 = first;
    c.tail = 0;
    return c;
  }
  c.g0 = first / kPer16 * kPer16;
  c.lead = static_cast<int>(first - c.g0);
  int64_t end = (first + count + kPer16 - 1) / kPer16 * kPer16;
  int64_t safe_end = total / kPer16 * kPer16;  // last full 16-byte chunk
  if (end > safe_end) end = safe_end > c.g0 ? safe_end : c.g0;
  c.bytes = static_cast<uint32_t>((end - c.g0) * E);
  c.tail0 = end;
  c.tail = static_cast<int>(first + count > end ? first + count - end : 0);
  return c;
}

}  // namespace tma

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
