// Gather-floor probe for CSR SpMV on sm_100a (measurement only; not part of
// the Sparse BLAS library and never called by it).
//
// A CSR SpMV over a matrix with random columns is bound by two streams that
// share the load/store path: the read-once column indices and values, and one
// random gather of x per nonzero.  These kernels time the two streams alone
// and together, with no row structure at all (one flat sum per thread), so
// they bound from below what any row-segmented kernel can reach on the same
// arrays:
//   mode 0  indices/values, 8 contiguous positions per lane, 16-byte loads
//           (the pattern of the register-segmented kernel), plus gathers
//   mode 1  the same with 32-byte loads (ld.global.*.v4.b64 / v8.b32)
//   mode 2  coalesced 16-byte loads (lane-interleaved), plus gathers
//   mode 3  gathers only; the column is a hash of the position
//   mode 4  indices/values only (mode 1's loads), no gather
// Gather flavours: 0 ld.global.nc, 1 ld.global.nc.L1::no_allocate,
// 2 ld.global.cg (L2 only).
// Every warp takes a contiguous run of 256-position tiles, as the
// register-segmented kernel does; each thread writes one partial sum.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kThreads = 128;
constexpr int kTile = 256;

template <int G>
__device__ __forceinline__ double gather(const double* p) {
  double v;
  if (G == 0) {
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
  } else if (G == 1) {
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  } else {
    asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p));
  }
  return v;
}

__device__ __forceinline__ void ld16(const int64_t* p, int64_t& a, int64_t& b) {
  asm volatile("ld.global.cs.v2.s64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}
__device__ __forceinline__ void ld16(const double* p, double& a, double& b) {
  asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "l"(p));
}
__device__ __forceinline__ void ld32(const int64_t* p, int64_t& a, int64_t& b, int64_t& c,
                                     int64_t& d) {
  asm volatile("ld.global.cs.v4.s64 {%0, %1, %2, %3}, [%4];"
               : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
}
__device__ __forceinline__ void ld32(const double* p, double& a, double& b, double& c,
                                     double& d) {
  asm volatile("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}

__device__ __forceinline__ uint64_t mix(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

template <int MODE, int G>
__global__ void __launch_bounds__(kThreads) flat_kernel(const int64_t* __restrict__ idx,
                                                        const double* __restrict__ val,
                                                        const double* __restrict__ x,
                                                        int64_t ntiles, int64_t n,
                                                        double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = static_cast<int64_t>(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5);
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kThreads / 32);
  const int64_t per = (ntiles + warps - 1) / warps;
  const int64_t tb = warp * per;
  const int64_t te = tb + per < ntiles ? tb + per : ntiles;
  double acc = 0.0;
  for (int64_t t = tb; t < te; ++t) {
    const int64_t base = t * kTile;
    int64_t c[8];
    double v[8];
    if (MODE == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        ld16(idx + base + 8 * lane + 2 * j, c[2 * j], c[2 * j + 1]);
        ld16(val + base + 8 * lane + 2 * j, v[2 * j], v[2 * j + 1]);
      }
    } else if (MODE == 1 || MODE == 4) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        ld32(idx + base + 8 * lane + 4 * j, c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]);
        ld32(val + base + 8 * lane + 4 * j, v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      }
    } else if (MODE == 2) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        ld16(idx + base + 64 * j + 2 * lane, c[2 * j], c[2 * j + 1]);
        ld16(val + base + 64 * j + 2 * lane, v[2 * j], v[2 * j + 1]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        c[k] = static_cast<int64_t>(mix(static_cast<uint64_t>(base + 8 * lane + k)) %
                                    static_cast<uint64_t>(n));
        v[k] = 1.0;
      }
    }
    if (MODE == 4) {
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += v[k] * static_cast<double>(c[k]);
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) acc += v[k] * gather<G>(x + c[k]);
    }
  }
  out[static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x] = acc;
}

template <int MODE>
int launch_mode(cudaStream_t s, int g, const int64_t* idx, const double* val, const double* x,
                int64_t ntiles, int64_t n, double* out, int blocks) {
  if (g == 0) flat_kernel<MODE, 0><<<blocks, kThreads, 0, s>>>(idx, val, x, ntiles, n, out);
  if (g == 1) flat_kernel<MODE, 1><<<blocks, kThreads, 0, s>>>(idx, val, x, ntiles, n, out);
  if (g == 2) flat_kernel<MODE, 2><<<blocks, kThreads, 0, s>>>(idx, val, x, ntiles, n, out);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace

// Threads per CTA of the probe kernels (the output holds one double per thread).
extern "C" __attribute__((visibility("default"))) int ascb_probe_threads(void) {
  return kThreads;
}

// One launch of probe `mode` with gather flavour `gather` over the first
// 256 * floor(nnz / 256) positions of idx / val (32-byte aligned) and x[n];
// `out` holds blocks * ascb_probe_threads() doubles.  Returns the launch's
// cudaError_t, or -1 for a bad argument.
extern "C" __attribute__((visibility("default"))) int ascb_probe_flat(
    void* stream, int mode, int gather, const int64_t* idx, const double* val, const double* x,
    int64_t nnz, int64_t n, double* out, int blocks) {
  if (mode < 0 || mode > 4 || gather < 0 || gather > 2 || blocks < 1 || n < 1) return -1;
  if (((reinterpret_cast<uintptr_t>(idx) | reinterpret_cast<uintptr_t>(val)) & 31u) != 0) return -1;
  const int64_t ntiles = nnz / kTile;
  auto s = static_cast<cudaStream_t>(stream);
  switch (mode) {
    case 0: return launch_mode<0>(s, gather, idx, val, x, ntiles, n, out, blocks);
    case 1: return launch_mode<1>(s, gather, idx, val, x, ntiles, n, out, blocks);
    case 2: return launch_mode<2>(s, gather, idx, val, x, ntiles, n, out, blocks);
    case 3: return launch_mode<3>(s, gather, idx, val, x, ntiles, n, out, blocks);
    default: return launch_mode<4>(s, gather, idx, val, x, ntiles, n, out, blocks);
  }
}
