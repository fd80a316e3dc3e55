// Sparse triangular solve op(A) X = alpha B on sm_100a, X overwriting the
// dense right-hand sides B (n x k, row or column major), for the CSR arrays of
// M = op(A) with sorted columns (the stored arrays for op = none, the stable
// transposed structure otherwise).  Contract: SparseTriangularSolve[Multiple]
// (include/asc/sparse/blas.h:1774-1910) and the CUDA facet's
// StandardTriangularSolveKernel (src/sparse/cuda/kernels.cu:349-391):
//   value = alpha * B(row); value -= M(row, c) * X(c) for the row's strict
//   triangle in increasing c; value /= M(row, row) unless the diagonal is
//   unit; X(row) = value.
//
// Synchronisation-free schedule (after Liu et al., "A Synchronization-Free
// Algorithm for Parallel Sparse Triangular Solves", Euro-Par 2016): one
// launch, persistent warps, each warp takes the next row in solve order from
// an atomic ticket, waits for the rows its entries depend on through per-row
// ready flags (acquire loads), solves the row and publishes it (release
// store).  Tickets are handed out in solve order, so every row a warp waits
// for belongs to a warp that is already running: the solve cannot deadlock
// whatever the grid or occupancy.  Every wait is bounded (time and polls);
// one that gives up raises an abort flag that releases all other waits and
// records 1 in the status word, so the kernel always ends.
//
// One right-hand side: lanes take 32 entries of the row at a time, wait and
// gather in parallel, form the products, and
//   EXACT (DETERMINISTIC): lane 0 subtracts them in stored order with
//     separately rounded operations -- the reference's arithmetic, bit for bit;
//   FAST (BACKEND_DEFAULT): lanes accumulate with FMA, one warp reduction
//     per row.
// Several right-hand sides: lanes take 32 right-hand sides at a time and walk
// the row's entries in stored order (exact in both modes).
// Complex division is Smith's method (Smith, CACM 5(8), 1962) in the order of
// the facet's DeviceArithmetic::Divide (kernels.cu:58-72).
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s per wait
constexpr uint32_t kMaxPolls = 1u << 26;

template <typename R>
struct Cx {
  R re, im;
};

__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

template <typename T>
struct Ar {  // real
  __device__ static T zero() { return T(0); }
  __device__ static T mul(T a, T b) { return mul_rn(a, b); }
  __device__ static T sub(T a, T b) { return sub_rn(a, b); }
  __device__ static T div(T a, T b) { return div_rn(a, b); }
  __device__ static T conj(T a) { return a; }
  __device__ static T fma_sub(T acc, T a, T b) { return fma(a, b, acc); }  // acc + a b
  __device__ static T shfl(T v, int src) { return __shfl_sync(kFull, v, src); }
  __device__ static T shfl_xor(T v, int m) { return __shfl_xor_sync(kFull, v, m); }
  __device__ static T add(T a, T b) { return a + b; }
  __device__ static T load_l2(const T* p) { return __ldcg(p); }
  __device__ static T load(const T* p) { return __ldg(p); }
};

template <typename R>
struct Ar<Cx<R>> {
  using T = Cx<R>;
  __device__ static T zero() { return {R(0), R(0)}; }
  __device__ static T mul(T a, T b) {
    return {sub_rn(mul_rn(a.re, b.re), mul_rn(a.im, b.im)),
            add_rn(mul_rn(a.re, b.im), mul_rn(a.im, b.re))};
  }
  __device__ static T sub(T a, T b) { return {sub_rn(a.re, b.re), sub_rn(a.im, b.im)}; }
  __device__ static T div(T n, T d) {
    const R adr = d.re < R(0) ? -d.re : d.re;
    const R adi = d.im < R(0) ? -d.im : d.im;
    if (adr >= adi) {
      const R ratio = div_rn(d.im, d.re);
      const R den = add_rn(d.re, mul_rn(d.im, ratio));
      return {div_rn(add_rn(n.re, mul_rn(n.im, ratio)), den),
              div_rn(sub_rn(n.im, mul_rn(n.re, ratio)), den)};
    }
    const R ratio = div_rn(d.re, d.im);
    const R den = add_rn(d.im, mul_rn(d.re, ratio));
    return {div_rn(add_rn(mul_rn(n.re, ratio), n.im), den),
            div_rn(sub_rn(mul_rn(n.im, ratio), n.re), den)};
  }
  __device__ static T conj(T a) { return {a.re, -a.im}; }
  __device__ static T fma_sub(T acc, T a, T b) {  // acc + a b
    return {fma(-a.im, b.im, fma(a.re, b.re, acc.re)), fma(a.im, b.re, fma(a.re, b.im, acc.im))};
  }
  __device__ static T shfl(T v, int src) {
    return {__shfl_sync(kFull, v.re, src), __shfl_sync(kFull, v.im, src)};
  }
  __device__ static T shfl_xor(T v, int m) {
    return {__shfl_xor_sync(kFull, v.re, m), __shfl_xor_sync(kFull, v.im, m)};
  }
  __device__ static T add(T a, T b) { return {a.re + b.re, a.im + b.im}; }
  __device__ static T load_l2(const T* p) {
    const R* q = reinterpret_cast<const R*>(p);
    return {__ldcg(q), __ldcg(q + 1)};
  }
  __device__ static T load(const T* p) {
    const R* q = reinterpret_cast<const R*>(p);
    return {__ldg(q), __ldg(q + 1)};
  }
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct Control {
  unsigned long long ticket;
  unsigned abort;
  unsigned pad;
};

// Waits until row c is published.  False if the wait gave up (or another
// wait did): the caller goes on with whatever X holds; the status word says
// the result is invalid.
__device__ bool wait_ready(const unsigned* ready, int64_t c, Control* ctl, int* status) {
  if (ld_acquire(ready + c) != 0u) return true;
  const uint64_t start = global_ns();
  for (uint32_t i = 1; i < kMaxPolls; ++i) {
    if (i > 32) __nanosleep(i > 4096 ? 256 : 32);
    if (ld_acquire(ready + c) != 0u) return true;
    if ((i & 63u) == 0u) {
      if (*reinterpret_cast<volatile unsigned*>(&ctl->abort) != 0u) return false;
      if (global_ns() - start > kWaitNs) break;
    }
  }
  atomicExch(&ctl->abort, 1u);
  if (status != nullptr) atomicExch(status, 1);
  return false;
}

__device__ __forceinline__ int64_t elem(int64_t r, int64_t j, int64_t ld, bool row_major) {
  return row_major ? r * ld + j : j * ld + r;
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(kThreads) trsv_rows(ascb_trsv a, T alpha) {
  using A = Ar<T>;
  const int lane = threadIdx.x & 31;
  const T* __restrict__ val = static_cast<const T*>(a.val);
  T* x = static_cast<T*>(a.x);
  unsigned* ready = a.ready;
  Control* ctl = reinterpret_cast<Control*>(a.control);
  const bool row_major = a.row_major != 0;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&ctl->ticket, 1ull);
    t = __shfl_sync(kFull, t, 0);
    if (t >= static_cast<unsigned long long>(a.n)) break;
    const int64_t row = a.lower ? static_cast<int64_t>(t) : a.n - 1 - static_cast<int64_t>(t);
    const int64_t beg = __ldg(a.ptr + row);
    const int64_t end = __ldg(a.ptr + row + 1);
    if (a.k == 1) {
      T value = A::zero();
      if (lane == 0) value = A::mul(alpha, A::load_l2(x + elem(row, 0, a.ld, row_major)));
      T acc = A::zero();  // FAST: this lane's sum of products
      T diag = A::zero();
      for (int64_t p0 = beg; p0 < end; p0 += 32) {
        const int64_t p = p0 + lane;
        bool in_tri = false;
        bool is_diag = false;
        T v = A::zero();
        T prod = A::zero();
        if (p < end) {
          const int64_t c = __ldg(a.idx + p);
          v = A::load(val + p);
          if (a.conj) v = A::conj(v);
          is_diag = c == row;
          in_tri = a.lower ? c < row : c > row;
          if (in_tri) {
            wait_ready(ready, c, ctl, a.status);
            const T xc = A::load_l2(x + elem(c, 0, a.ld, row_major));
            if (EXACT) {
              prod = A::mul(v, xc);
            } else {
              acc = A::fma_sub(acc, v, xc);
            }
          }
        }
        const unsigned dmask = __ballot_sync(kFull, is_diag);
        if (dmask != 0u) diag = A::shfl(v, __ffs(dmask) - 1);
        if (EXACT) {
          unsigned mask = __ballot_sync(kFull, in_tri);
          while (mask != 0u) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1u;
            const T pk = A::shfl(prod, src);
            if (lane == 0) value = A::sub(value, pk);
          }
        }
      }
      if (!EXACT) {
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) acc = A::add(acc, A::shfl_xor(acc, m));
        if (lane == 0) value = A::sub(value, acc);
      }
      if (lane == 0) {
        if (!a.unit) value = A::div(value, diag);
        x[elem(row, 0, a.ld, row_major)] = value;
        st_release(ready + row, 1u);
      }
      continue;
    }
    // several right-hand sides: lane j of group j0 owns X(row, j0 + j)
    for (int64_t j0 = 0; j0 < a.k; j0 += 32) {
      const int64_t j = j0 + lane;
      const bool active = j < a.k;
      T value = A::zero();
      if (active) value = A::mul(alpha, A::load_l2(x + elem(row, j, a.ld, row_major)));
      T diag = A::zero();
      for (int64_t p0 = beg; p0 < end; p0 += 32) {
        const int64_t p = p0 + lane;
        int64_t c = -1;
        T v = A::zero();
        bool in_tri = false;
        if (p < end) {
          c = __ldg(a.idx + p);
          v = A::load(val + p);
          if (a.conj) v = A::conj(v);
          in_tri = a.lower ? c < row : c > row;
          if (in_tri && j0 == 0) wait_ready(ready, c, ctl, a.status);
        }
        __syncwarp();
        const unsigned dmask = __ballot_sync(kFull, p < end && c == row);
        if (dmask != 0u) diag = A::shfl(v, __ffs(dmask) - 1);
        unsigned mask = __ballot_sync(kFull, in_tri);
        while (mask != 0u) {
          // up to four entries at a time: their loads overlap, the
          // subtractions stay in stored order
          int src[4];
          int cnt = 0;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            src[u] = mask != 0u ? __ffs(mask) - 1 : -1;
            if (mask != 0u) {
              mask &= mask - 1u;
              ++cnt;
            }
          }
          T xv[4];
          T vv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int s = src[u] < 0 ? 0 : src[u];
            const int64_t cu = __shfl_sync(kFull, c, s);
            vv[u] = A::shfl(v, s);
            xv[u] = (u < cnt && active) ? A::load_l2(x + elem(cu, j, a.ld, row_major)) : A::zero();
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (u < cnt && active) value = A::sub(value, A::mul(vv[u], xv[u]));
          }
        }
      }
      if (active) {
        if (!a.unit) value = A::div(value, diag);
        x[elem(row, j, a.ld, row_major)] = value;
      }
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release(ready + row, 1u);
  }
}

template <typename T>
__global__ void dense_zero(T* x, int64_t rows, int64_t cols, int64_t ld, bool row_major) {
  const int64_t total = rows * cols;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += step) {
    const int64_t r = e % rows;
    const int64_t j = e / rows;
    x[elem(r, j, ld, row_major)] = Ar<T>::zero();
  }
}

template <typename T, bool EXACT>
int launch_rows(cudaStream_t s, const ascb_trsv& a, T alpha, int sm) {
  static int per_sm = 0;
  if (per_sm == 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, trsv_rows<T, EXACT>, kThreads, 0) !=
            cudaSuccess ||
        b <= 0) {
      b = 1;
    }
    per_sm = b;
  }
  const int64_t warps_needed = a.n;
  int64_t blocks = static_cast<int64_t>(sm > 0 ? sm : 148) * per_sm;
  const int64_t need = (warps_needed + kThreads / 32 - 1) / (kThreads / 32);
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  trsv_rows<T, EXACT><<<static_cast<unsigned>(blocks), kThreads, 0, s>>>(a, alpha);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int run(cudaStream_t s, int exact, const ascb_trsv& a, T alpha, int sm) {
  if (cudaMemsetAsync(a.control, 0, ascb_trsv_scratch_bytes(a.n), s) != cudaSuccess) {
    return static_cast<int>(cudaGetLastError());
  }
  return exact ? launch_rows<T, true>(s, a, alpha, sm) : launch_rows<T, false>(s, a, alpha, sm);
}

template <typename T>
int zero(cudaStream_t s, const ascb_trsv& a, int sm) {
  const int64_t total = a.n * a.k;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  dense_zero<T><<<static_cast<unsigned>(blocks), 256, 0, s>>>(static_cast<T*>(a.x), a.n, a.k,
                                                              a.ld, a.row_major != 0);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace ascb

extern "C" size_t ascb_trsv_scratch_bytes(int64_t n) {
  // Control block (ticket, abort) and then one ready flag per row; the ready
  // flags start 16 bytes in.
  return 16 + static_cast<size_t>(n > 0 ? n : 0) * sizeof(unsigned);
}

extern "C" int ascb_sptrsv(void* stream, int dtype, int exact, int alpha_is_zero,
                           const ascb_trsv* t, double alpha_re, double alpha_im, int sm_count) {
  using namespace ascb;
  auto s = static_cast<cudaStream_t>(stream);
  if (t->n <= 0 || t->k <= 0) return 0;
  switch (dtype) {
    case ASCB_F64:
      return alpha_is_zero ? zero<double>(s, *t, sm_count)
                           : run<double>(s, exact, *t, alpha_re, sm_count);
    case ASCB_F32:
      return alpha_is_zero ? zero<float>(s, *t, sm_count)
                           : run<float>(s, exact, *t, static_cast<float>(alpha_re), sm_count);
    case ASCB_C128:
      return alpha_is_zero ? zero<Cx<double>>(s, *t, sm_count)
                           : run<Cx<double>>(s, exact, *t, Cx<double>{alpha_re, alpha_im},
                                             sm_count);
    case ASCB_C64:
      return alpha_is_zero
                 ? zero<Cx<float>>(s, *t, sm_count)
                 : run<Cx<float>>(s, exact, *t,
                                  Cx<float>{static_cast<float>(alpha_re),
                                            static_cast<float>(alpha_im)},
                                  sm_count);
    default:
      return static_cast<int>(cudaErrorInvalidValue);
  }
}
