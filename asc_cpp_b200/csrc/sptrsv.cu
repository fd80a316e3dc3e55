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
// Schedule: one launch, persistent warps, synchronisation free (Liu et al.,
// Euro-Par 2016; thread-level rows as in Su et al., "CapelliniSpTRSV",
// HPDC 2020).  Rows are taken in a topological "solve order" -- increasing
// rows for lower M, decreasing for upper M, or the level order of an analysis
// (asc_sb_plan_triangular_analysis) -- in groups of 32 from an atomic ticket.
// Every row a group depends on is either in an earlier group, whose warp is
// already running, or earlier in the same group, so the solve cannot deadlock
// whatever the grid.
//
// One right-hand side, short rows: lane i owns the group's i-th row and walks
// its entries in stored order.  A dependency inside the group is read from
// shared memory once the owning lane has finished (ballot mask); one outside
// is read from the published-value array, which holds a signalling-NaN
// sentinel until the row is solved.  Arithmetic never produces that bit
// pattern (it returns the canonical NaN), so the value itself is the ready
// flag: no separate flag, no fence on the critical path.  Groups with a row
// longer than kLongRow entries are solved row after row by the whole warp
// (lanes over entries).  Several right-hand sides: rows of a group one after
// the other, lanes over right-hand sides, per-row ready flags (release /
// acquire).
//
// EXACT (DETERMINISTIC): every product and difference rounded separately in
// stored order -- the reference's arithmetic, bit for bit.  FAST
// (BACKEND_DEFAULT): the lane path fuses each product and difference (FMA);
// the warp path sums with FMA and one reduction per row.  Both are the same
// every run.  Complex division is Smith's method (Smith, CACM 5(8), 1962) in
// the order of the facet's DeviceArithmetic::Divide (kernels.cu:58-72).
//
// Every wait is bounded (the context's wait limit, 2 s by default, and a poll
// count); one that gives up raises an abort flag that ends all other waits
// and records 1 in the status word.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

// Launch and polling shape (compile-time; the defaults are the measured best
// on B200).  Row order keeps as many warps in flight as fit: its groups chain
// through their neighbours, and wavefronts need a wide window of rows.  Level
// order already puts whole levels side by side; there fewer polling warps
// shorten every hand-over between levels (1 CTA per SM: 4.0 ms against
// 10.4 ms at full occupancy on the lower triangle of a 1000 x 1000 5-point
// Laplacian).
#ifndef ASCB_TRSV_CTAS_PER_SM
#define ASCB_TRSV_CTAS_PER_SM 0  // row order; 0: as many as fit
#endif
#ifndef ASCB_TRSV_LEVEL_CTAS_PER_SM
#define ASCB_TRSV_LEVEL_CTAS_PER_SM 1  // level order
#endif
#ifndef ASCB_TRSV_IDLE_SPIN
#define ASCB_TRSV_IDLE_SPIN 32  // idle warp iterations before backing off
#endif
#ifndef ASCB_TRSV_SLEEP_NS
#define ASCB_TRSV_SLEEP_NS 32  // back-off per idle iteration
#endif

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int64_t kLongRow = 64;
constexpr uint64_t kWaitNs = 2000000000ull;
constexpr uint32_t kMaxPolls = 1u << 26;

template <typename R>
struct Cx {
  R re, im;
};

__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// ---- published values: relaxed gpu-scope accesses, sNaN sentinel ----------
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
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

template <typename R>
struct Bits;
template <>
struct Bits<double> {
  using U = uint64_t;
  static constexpr U kSentinel = 0x7ff0000000000001ull;  // a signalling NaN
  __device__ static U to(double v) { return static_cast<U>(__double_as_longlong(v)); }
  __device__ static double from(U u) { return __longlong_as_double(static_cast<long long>(u)); }
};
template <>
struct Bits<float> {
  using U = uint32_t;
  static constexpr U kSentinel = 0x7f800001u;  // a signalling NaN
  __device__ static U to(float v) { return __float_as_uint(v); }
  __device__ static float from(U u) { return __uint_as_float(u); }
};

template <typename T>
struct Ar {  // real element arithmetic
  using R = T;
  static constexpr int kParts = 1;
  __device__ static T zero() { return T(0); }
  __device__ static T mul(T a, T b) { return mul_rn(a, b); }
  __device__ static T sub(T a, T b) { return sub_rn(a, b); }
  __device__ static T div(T a, T b) { return div_rn(a, b); }
  __device__ static T conj(T a) { return a; }
  __device__ static T fma_acc(T acc, T a, T b) { return fma(a, b, acc); }        // acc + a b
  __device__ static T fms(T value, T a, T b) { return fma(-a, b, value); }       // value - a b
  __device__ static T shfl(T v, int src) { return __shfl_sync(kFull, v, src); }
  __device__ static T shfl_xor(T v, int m) { return __shfl_xor_sync(kFull, v, m); }
  __device__ static T add(T a, T b) { return a + b; }
  __device__ static T load(const T* p) { return __ldg(p); }
  __device__ static T load_l2(const T* p) { return __ldcg(p); }
  // published value of row c, or false while it is the sentinel
  __device__ static bool poll(const T* pub, T* out) {
    using B = Bits<T>;
    const auto u = ld_relaxed(reinterpret_cast<const typename B::U*>(pub));
    if (u == B::kSentinel) return false;
    *out = B::from(u);
    return true;
  }
  __device__ static void publish(T* pub, T v) {
    using B = Bits<T>;
    st_relaxed(reinterpret_cast<typename B::U*>(pub), B::to(v));
  }
  __device__ static void sentinel(T* pub) {
    *reinterpret_cast<typename Bits<T>::U*>(pub) = Bits<T>::kSentinel;
  }
};

template <typename Rl>
struct Ar<Cx<Rl>> {
  using R = Rl;
  using T = Cx<Rl>;
  static constexpr int kParts = 2;
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
  __device__ static T fma_acc(T acc, T a, T b) {
    return {fma(-a.im, b.im, fma(a.re, b.re, acc.re)), fma(a.im, b.re, fma(a.re, b.im, acc.im))};
  }
  __device__ static T fms(T v, T a, T b) {
    return {fma(a.im, b.im, fma(-a.re, b.re, v.re)), fma(-a.im, b.re, fma(-a.re, b.im, v.im))};
  }
  __device__ static T shfl(T v, int src) {
    return {__shfl_sync(kFull, v.re, src), __shfl_sync(kFull, v.im, src)};
  }
  __device__ static T shfl_xor(T v, int m) {
    return {__shfl_xor_sync(kFull, v.re, m), __shfl_xor_sync(kFull, v.im, m)};
  }
  __device__ static T add(T a, T b) { return {a.re + b.re, a.im + b.im}; }
  __device__ static T load(const T* p) {
    const R* q = reinterpret_cast<const R*>(p);
    return {__ldg(q), __ldg(q + 1)};
  }
  __device__ static T load_l2(const T* p) {
    const R* q = reinterpret_cast<const R*>(p);
    return {__ldcg(q), __ldcg(q + 1)};
  }
  // the two parts are published by separate stores; the value is ready
  // once neither is the sentinel (each part is written once)
  __device__ static bool poll(const T* pub, T* out) {
    using B = Bits<R>;
    const auto* q = reinterpret_cast<const typename B::U*>(pub);
    const auto re = ld_relaxed(q);
    if (re == B::kSentinel) return false;
    const auto im = ld_relaxed(q + 1);
    if (im == B::kSentinel) return false;
    *out = {B::from(re), B::from(im)};
    return true;
  }
  __device__ static void publish(T* pub, T v) {
    using B = Bits<R>;
    auto* q = reinterpret_cast<typename B::U*>(pub);
    st_relaxed(q, B::to(v.re));
    st_relaxed(q + 1, B::to(v.im));
  }
  __device__ static void sentinel(T* pub) {
    auto* q = reinterpret_cast<typename Bits<R>::U*>(pub);
    q[0] = Bits<R>::kSentinel;
    q[1] = Bits<R>::kSentinel;
  }
};

struct Control {
  unsigned long long ticket;
  unsigned abort;
  unsigned pad;
};

__device__ __forceinline__ bool aborted(const Control* ctl) {
  return *reinterpret_cast<const volatile unsigned*>(&ctl->abort) != 0u;
}
__device__ __noinline__ void give_up(Control* ctl, int* status) {
  atomicExch(&ctl->abort, 1u);
  if (status != nullptr) atomicExch(status, 1);
}

// Bounded spin until `ready()` holds.  False if this wait or another one gave
// up; the caller goes on and the status word marks the result invalid.
template <typename F>
__device__ bool bounded_wait(F ready, Control* ctl, int* status, uint64_t limit_ns) {
  if (ready()) return true;
  const uint64_t start = global_ns();
  for (uint32_t i = 1; i < kMaxPolls; ++i) {
    if (i > 32) __nanosleep(i > 4096 ? 256 : 32);
    if (ready()) return true;
    if ((i & 63u) == 0u) {
      if (aborted(ctl)) return false;
      if (global_ns() - start > limit_ns) break;
    }
  }
  give_up(ctl, status);
  return false;
}

// The wait limit of a solve: the context's setting, else kWaitNs.
__device__ __forceinline__ uint64_t wait_limit(const ascb_trsv& a) {
  return a.wait_ns != 0 ? a.wait_ns : kWaitNs;
}

__device__ __forceinline__ int64_t elem(int64_t r, int64_t j, int64_t ld, bool row_major) {
  return row_major ? r * ld + j : j * ld + r;
}
// Row at solve position s, and solve position of row r.
__device__ __forceinline__ int64_t row_at(const ascb_trsv& a, int64_t s) {
  return a.order != nullptr ? __ldg(a.order + s) : (a.lower ? s : a.n - 1 - s);
}
__device__ __forceinline__ int64_t position_of(const ascb_trsv& a, int64_t r) {
  return a.position != nullptr ? __ldg(a.position + r) : (a.lower ? r : a.n - 1 - r);
}
__device__ __forceinline__ bool outside(const ascb_trsv& a, int64_t c, int64_t row) {
  return a.lower ? c > row : c < row;
}

__device__ __forceinline__ unsigned long long take_ticket(Control* ctl, int lane) {
  unsigned long long t = 0;
  if (lane == 0) t = atomicAdd(&ctl->ticket, 1ull);
  return __shfl_sync(kFull, t, 0);
}

// One row by the whole warp (lanes over entries); dependencies from the
// published values.  Lane 0 ends with the row's value.
template <typename T, bool EXACT>
__device__ void warp_row(const ascb_trsv& a, int64_t row, T alpha, T* pub, Control* ctl,
                         int lane, T* stage) {
  using A = Ar<T>;
  const T* __restrict__ val = static_cast<const T*>(a.val);
  T* x = static_cast<T*>(a.x);
  const int64_t beg = __ldg(a.ptr + row);
  const int64_t end = __ldg(a.ptr + row + 1);
  T value = A::zero();
  if (lane == 0) value = A::mul(alpha, x[elem(row, 0, a.ld, a.row_major != 0)]);
  T acc = A::zero();
  T diag = A::zero();
  for (int64_t p0 = beg; p0 < end; p0 += 32) {
    const int64_t p = p0 + lane;
    bool dep = false;
    bool is_diag = false;
    T v = A::zero();
    T prod = A::zero();
    if (p < end) {
      const int64_t c = __ldg(a.idx + p);
      v = A::load(val + p);
      if (a.conj) v = A::conj(v);
      is_diag = c == row;
      dep = !is_diag && !outside(a, c, row);
      if (dep) {
        T xc = A::zero();
        bounded_wait([&] { return A::poll(pub + c, &xc); }, ctl, a.status, wait_limit(a));
        if (EXACT) {
          prod = A::mul(v, xc);
        } else {
          acc = A::fma_acc(acc, v, xc);
        }
      }
    }
    const unsigned dmask = __ballot_sync(kFull, is_diag);
    if (dmask != 0u) diag = A::shfl(v, __ffs(dmask) - 1);
    if (EXACT) {
      // the chunk's dependencies are contiguous lanes (sorted columns): lane 0
      // subtracts their products in stored order from shared memory
      const unsigned mask = __ballot_sync(kFull, dep);
      if (mask != 0u) {
        stage[lane] = prod;
        __syncwarp();
        if (lane == 0) {
          const int first = __ffs(mask) - 1;
          const int last = 31 - __clz(mask);
          for (int q = first; q <= last; ++q) {
            if ((mask >> q) & 1u) value = A::sub(value, stage[q]);
          }
        }
        __syncwarp();
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
    x[elem(row, 0, a.ld, a.row_major != 0)] = value;
    A::publish(pub + row, value);
  }
  __syncwarp();
}

// One right-hand side.
template <typename T, bool EXACT>
__global__ void __launch_bounds__(kThreads) trsv_single(ascb_trsv a, T alpha) {
  using A = Ar<T>;
  __shared__ T solved_value[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const T* __restrict__ val = static_cast<const T*>(a.val);
  T* x = static_cast<T*>(a.x);
  T* pub = static_cast<T*>(a.pub);
  Control* ctl = static_cast<Control*>(a.control);
  const bool row_major = a.row_major != 0;
  for (;;) {
    const unsigned long long t = take_ticket(ctl, lane);
    const int64_t s0 = static_cast<int64_t>(t) * 32;
    if (s0 >= a.n) break;
    const int64_t s = s0 + lane;
    const bool valid = s < a.n;
    const int64_t row = valid ? row_at(a, s) : 0;
    int64_t p = valid ? __ldg(a.ptr + row) : 0;
    const int64_t end = valid ? __ldg(a.ptr + row + 1) : 0;
    if (__any_sync(kFull, end - p > kLongRow)) {
      const int64_t count = a.n - s0 < 32 ? a.n - s0 : 32;
      for (int64_t i = 0; i < count; ++i) {
        warp_row<T, EXACT>(a, __shfl_sync(kFull, row, static_cast<int>(i)), alpha, pub, ctl, lane,
                           solved_value[warp]);
      }
      continue;
    }
    T value = valid ? A::mul(alpha, x[elem(row, 0, a.ld, row_major)]) : A::zero();
    T diag = A::zero();
    bool done = !valid;
    unsigned solved = 0u;  // lanes whose row is solved
    uint32_t idle = 0;
    uint64_t idle_since = 0;
    for (;;) {
      bool progressed = false;
      if (!done) {
        while (p < end) {
          const int64_t c = __ldg(a.idx + p);
          T v = A::load(val + p);
          if (a.conj) v = A::conj(v);
          if (c == row) {
            diag = v;
            ++p;
            continue;
          }
          if (outside(a, c, row)) {
            ++p;
            continue;
          }
          T xc;
          const int64_t sc = position_of(a, c);
          if (sc >= s0 && sc < s0 + 32) {  // earlier lane of this group
            const int li = static_cast<int>(sc - s0);
            if (((solved >> li) & 1u) == 0u) break;
            xc = solved_value[warp][li];
          } else if (!A::poll(pub + c, &xc)) {
            break;
          }
          value = EXACT ? A::sub(value, A::mul(v, xc)) : A::fms(value, v, xc);
          ++p;
          progressed = true;
        }
        if (p >= end) {
          if (!a.unit) value = A::div(value, diag);
          solved_value[warp][lane] = value;
          x[elem(row, 0, a.ld, row_major)] = value;
          A::publish(pub + row, value);
          done = true;
          progressed = true;
        }
      }
      __syncwarp();
      solved = __ballot_sync(kFull, done);
      if (solved == kFull) break;
      if (__any_sync(kFull, progressed)) {
        idle = 0;
        continue;
      }
      // every pending lane waits for a row of an earlier group
      if (idle == 0) idle_since = global_ns();
      ++idle;
      if (idle > ASCB_TRSV_IDLE_SPIN) __nanosleep(idle > 4096 ? 256 : ASCB_TRSV_SLEEP_NS);
      if ((idle & 63u) == 0u) {
        bool stop = aborted(ctl);
        if (!stop && (global_ns() - idle_since > wait_limit(a) || idle >= kMaxPolls)) {
          if (lane == 0) give_up(ctl, a.status);
          stop = true;
        }
        if (__any_sync(kFull, stop)) break;
      }
    }
  }
}

// Several right-hand sides: the group's rows one after the other, lane j of
// group j0 owns X(row, j0 + j); per-row ready flags.
template <typename T, bool EXACT>
__global__ void __launch_bounds__(kThreads) trsv_multi(ascb_trsv a, T alpha) {
  using A = Ar<T>;
  const int lane = threadIdx.x & 31;
  const T* __restrict__ val = static_cast<const T*>(a.val);
  T* x = static_cast<T*>(a.x);
  unsigned* ready = static_cast<unsigned*>(a.pub);
  Control* ctl = static_cast<Control*>(a.control);
  const bool row_major = a.row_major != 0;
  for (;;) {
    const unsigned long long t = take_ticket(ctl, lane);
    const int64_t s0 = static_cast<int64_t>(t) * 32;
    if (s0 >= a.n) break;
    const int64_t count = a.n - s0 < 32 ? a.n - s0 : 32;
    for (int64_t i = 0; i < count; ++i) {
      const int64_t row = row_at(a, s0 + i);
      const int64_t beg = __ldg(a.ptr + row);
      const int64_t end = __ldg(a.ptr + row + 1);
      for (int64_t j0 = 0; j0 < a.k; j0 += 32) {
        const int64_t j = j0 + lane;
        const bool active = j < a.k;
        T value = A::zero();
        if (active) value = A::mul(alpha, x[elem(row, j, a.ld, row_major)]);
        T diag = A::zero();
        for (int64_t p0 = beg; p0 < end; p0 += 32) {
          const int64_t p = p0 + lane;
          int64_t c = -1;
          T v = A::zero();
          bool dep = false;
          if (p < end) {
            c = __ldg(a.idx + p);
            v = A::load(val + p);
            if (a.conj) v = A::conj(v);
            dep = c != row && !outside(a, c, row);
            if (dep && j0 == 0) {
              bounded_wait([&] { return ld_acquire(ready + c) != 0u; }, ctl, a.status, wait_limit(a));
            }
          }
          __syncwarp();
          const unsigned dmask = __ballot_sync(kFull, p < end && c == row);
          if (dmask != 0u) diag = A::shfl(v, __ffs(dmask) - 1);
          unsigned mask = __ballot_sync(kFull, dep);
          while (mask != 0u) {
            // up to four entries at a time: their loads overlap, the
            // differences stay in stored order
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
              const int sl = src[u] < 0 ? 0 : src[u];
              const int64_t cu = __shfl_sync(kFull, c, sl);
              vv[u] = A::shfl(v, sl);
              xv[u] = (u < cnt && active) ? A::load_l2(x + elem(cu, j, a.ld, row_major))
                                          : A::zero();
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              if (u < cnt && active) {
                value = EXACT ? A::sub(value, A::mul(vv[u], xv[u])) : A::fms(value, vv[u], xv[u]);
              }
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
      __syncwarp();
    }
  }
}

// Clears the control block and marks every row unsolved.
template <typename T>
__global__ void trsv_prepare(ascb_trsv a) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (first == 0) {
    Control* ctl = static_cast<Control*>(a.control);
    ctl->ticket = 0ull;
    ctl->abort = 0u;
  }
  if (a.k == 1) {
    T* pub = static_cast<T*>(a.pub);
    for (int64_t r = first; r < a.n; r += step) Ar<T>::sentinel(pub + r);
  } else {
    unsigned* ready = static_cast<unsigned*>(a.pub);
    for (int64_t r = first; r < a.n; r += step) ready[r] = 0u;
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

// ---- level analysis ---------------------------------------------------------
// level[r] = 1 + max level of the rows r depends on (1 for none), in the
// lane-per-row schedule above with integer maxima (order does not matter);
// level[] doubles as the ready flag (0 = unknown).  control->pad receives
// nothing; the caller sorts rows by level.
__global__ void __launch_bounds__(kThreads) trsv_levels(ascb_trsv a, int64_t* level) {
  __shared__ int64_t solved_level[kWarps][32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  Control* ctl = static_cast<Control*>(a.control);
  auto* lv = reinterpret_cast<uint64_t*>(level);
  for (;;) {
    const unsigned long long t = take_ticket(ctl, lane);
    const int64_t s0 = static_cast<int64_t>(t) * 32;
    if (s0 >= a.n) break;
    const int64_t s = s0 + lane;
    const bool valid = s < a.n;
    const int64_t row = valid ? (a.lower ? s : a.n - 1 - s) : 0;
    int64_t p = valid ? __ldg(a.ptr + row) : 0;
    const int64_t end = valid ? __ldg(a.ptr + row + 1) : 0;
    int64_t mine = 1;
    bool done = !valid;
    unsigned solved = 0u;
    uint32_t idle = 0;
    uint64_t idle_since = 0;
    for (;;) {
      bool progressed = false;
      if (!done) {
        while (p < end) {
          const int64_t c = __ldg(a.idx + p);
          if (c == row || outside(a, c, row)) {
            ++p;
            continue;
          }
          const int64_t sc = a.lower ? c : a.n - 1 - c;
          int64_t lc;
          if (sc >= s0 && sc < s0 + 32) {
            const int li = static_cast<int>(sc - s0);
            if (((solved >> li) & 1u) == 0u) break;
            lc = solved_level[warp][li];
          } else {
            lc = static_cast<int64_t>(ld_relaxed(lv + c));
            if (lc == 0) break;
          }
          if (lc + 1 > mine) mine = lc + 1;
          ++p;
          progressed = true;
        }
        if (p >= end) {
          solved_level[warp][lane] = mine;
          st_relaxed(lv + row, static_cast<uint64_t>(mine));
          done = true;
          progressed = true;
        }
      }
      __syncwarp();
      solved = __ballot_sync(kFull, done);
      if (solved == kFull) break;
      if (__any_sync(kFull, progressed)) {
        idle = 0;
        continue;
      }
      if (idle == 0) idle_since = global_ns();
      ++idle;
      if (idle > ASCB_TRSV_IDLE_SPIN) __nanosleep(idle > 4096 ? 256 : ASCB_TRSV_SLEEP_NS);
      if ((idle & 63u) == 0u) {
        bool stop = aborted(ctl);
        if (!stop && (global_ns() - idle_since > wait_limit(a) || idle >= kMaxPolls)) {
          if (lane == 0) give_up(ctl, a.status);
          stop = true;
        }
        if (__any_sync(kFull, stop)) break;
      }
    }
  }
}

__global__ void trsv_clear_levels(ascb_trsv a, int64_t* level) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (first == 0) {
    Control* ctl = static_cast<Control*>(a.control);
    ctl->ticket = 0ull;
    ctl->abort = 0u;
  }
  for (int64_t r = first; r < a.n; r += step) level[r] = 0;
}

__global__ void invert_order(const int64_t* order, int64_t n, int64_t* position) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < n; s += step) {
    position[order[s]] = s;
  }
}

unsigned GridFor(int64_t work, int threads, int sm, int per_sm) {
  int64_t blocks = (work + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return static_cast<unsigned>(blocks);
}

template <typename K>
int Resident(K kernel) {
  if (ASCB_TRSV_CTAS_PER_SM > 0) return ASCB_TRSV_CTAS_PER_SM;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kThreads, 0) != cudaSuccess ||
      b <= 0) {
    (void)cudaGetLastError();
    b = 1;
  }
  return b;
}

template <typename T, bool EXACT>
int launch_solve(cudaStream_t s, const ascb_trsv& a, T alpha, int sm) {
  trsv_prepare<T><<<GridFor(a.n, 256, sm, 8), 256, 0, s>>>(a);
  const int64_t groups = (a.n + 31) / 32;
  const bool levels = a.order != nullptr;
  if (a.k == 1) {
    static const int per_sm = Resident(trsv_single<T, EXACT>);
    const int use = levels ? ASCB_TRSV_LEVEL_CTAS_PER_SM : per_sm;
    trsv_single<T, EXACT><<<GridFor(groups, kWarps, sm, use), kThreads, 0, s>>>(a, alpha);
  } else {
    static const int per_sm = Resident(trsv_multi<T, EXACT>);
    const int use = levels ? ASCB_TRSV_LEVEL_CTAS_PER_SM : per_sm;
    trsv_multi<T, EXACT><<<GridFor(groups, kWarps, sm, use), kThreads, 0, s>>>(a, alpha);
  }
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int run(cudaStream_t s, int exact, const ascb_trsv& a, T alpha, int sm) {
  return exact ? launch_solve<T, true>(s, a, alpha, sm) : launch_solve<T, false>(s, a, alpha, sm);
}

template <typename T>
int zero(cudaStream_t s, const ascb_trsv& a, int sm) {
  dense_zero<T><<<GridFor(a.n * a.k, 256, sm, 8), 256, 0, s>>>(static_cast<T*>(a.x), a.n, a.k,
                                                               a.ld, a.row_major != 0);
  return static_cast<int>(cudaGetLastError());
}

}  // namespace
}  // namespace ascb

extern "C" size_t ascb_trsv_scratch_bytes(int64_t n, int elem_bytes) {
  // control block (16 bytes), then the published values (one right-hand
  // side) or the ready flags (several)
  const size_t per = elem_bytes > 4 ? static_cast<size_t>(elem_bytes) : 4;
  return 16 + static_cast<size_t>(n > 0 ? n : 0) * per;
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

extern "C" size_t ascb_trsv_analysis_bytes(int64_t n) {
  const size_t nn = static_cast<size_t>(n > 0 ? n : 0);
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  // level, order, position, bucket offsets, sort workspace
  return up(nn * 8) * 3 + up((nn + 2) * 8) + up(ascb_sort_workspace_bytes(n, n + 1));
}

extern "C" int ascb_trsv_analysis(void* stream, const ascb_trsv* t, void* workspace,
                                  int64_t** order, int64_t** position, int sm_count) {
  using namespace ascb;
  auto s = static_cast<cudaStream_t>(stream);
  const int64_t n = t->n;
  const size_t nn = static_cast<size_t>(n > 0 ? n : 0);
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  auto* ws = static_cast<unsigned char*>(workspace);
  auto* level = reinterpret_cast<int64_t*>(ws);
  auto* ord = reinterpret_cast<int64_t*>(ws + up(nn * 8));
  auto* pos = reinterpret_cast<int64_t*>(ws + 2 * up(nn * 8));
  auto* offsets = reinterpret_cast<int64_t*>(ws + 3 * up(nn * 8));
  void* sort_ws = ws + 3 * up(nn * 8) + up((nn + 2) * 8);
  *order = ord;
  *position = pos;
  if (n <= 0) return 0;
  ascb_trsv a = *t;
  a.order = nullptr;
  a.position = nullptr;
  trsv_clear_levels<<<GridFor(n, 256, sm_count, 8), 256, 0, s>>>(a, level);
  static const int per_sm = Resident(trsv_levels);
  trsv_levels<<<GridFor((n + 31) / 32, kWarps, sm_count, per_sm), kThreads, 0, s>>>(a, level);
  int e = static_cast<int>(cudaGetLastError());
  if (e != 0) return e;
  // stable by row within a level: rows of one level in increasing order
  e = ascb_stable_sort(stream, level, 1, n, n + 1, offsets, ord, sort_ws);
  if (e != 0) return e;
  invert_order<<<GridFor(n, 256, sm_count, 8), 256, 0, s>>>(ord, n, pos);
  return static_cast<int>(cudaGetLastError());
}
