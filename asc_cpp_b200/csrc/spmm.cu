// CSR x dense (SpMM) and the scatter (transpose) products, sm_100a.
//
// Row-major right-hand sides with 16-byte aligned rows take the chunked
// kernel below (one vector load per lane per stored entry).  Otherwise, for
// row-major right-hand sides:
// a group of G lanes owns one output row o and the lanes split its k columns,
// so each stored entry (o, c, v) costs one broadcast load of (c, v) and one
// coalesced load of the row B(c, :).  Each lane adds its columns' terms in
// stored order,
//     C(o, j) = C(o, j) + (alpha * v) * B(c, j),
// exactly the per-entry update of asc::Spmm (include/asc/sparse/blas.h:
// 1736-1748), with every product and sum rounded separately -- so this kernel
// is bit-exact against the serial reference and needs no separate
// deterministic variant.
//
// Other layouts fall back to one thread per output element (same arithmetic).
// Transposed products that have no transposed structure at hand scatter with
// atomics (BACKEND_DEFAULT only; order-dependent rounding within the bound).
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kThreads = 256;
constexpr int kEntryUnroll = 4;

// G lanes per row, J columns per lane (G*J >= k handled by an outer loop).
template <typename T, int G, int J>
__global__ void __launch_bounds__(kThreads)
spmm_row_major_kernel(int64_t rows, int64_t k, const int64_t* __restrict__ ptr,
                      const int64_t* __restrict__ idx, const T* __restrict__ val,
                      const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                      int64_t ldc, T alpha) {
  constexpr int kGroups = kThreads / G;
  const int lane = threadIdx.x % G;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * kGroups + threadIdx.x / G;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kGroups;
  for (int64_t o = first; o < rows; o += step) {
    const int64_t pb = __ldg(ptr + o);
    const int64_t pe = __ldg(ptr + o + 1);
    for (int64_t j0 = 0; j0 < k; j0 += int64_t{G} * J) {
      T acc[J];
      bool live[J];
#pragma unroll
      for (int t = 0; t < J; ++t) {
        const int64_t j = j0 + t * G + lane;
        live[t] = j < k;
        acc[t] = live[t] ? c[o * ldc + j] : T(0);
      }
      int64_t q = pb;
      for (; q + kEntryUnroll <= pe; q += kEntryUnroll) {
        int64_t col[kEntryUnroll];
        T av[kEntryUnroll];
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
          col[u] = __ldg(idx + q + u);
          av[u] = mul_rn(alpha, __ldg(val + q + u));
        }
        T bv[kEntryUnroll][J];
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
#pragma unroll
          for (int t = 0; t < J; ++t) {
            const int64_t j = j0 + t * G + lane;
            bv[u][t] = live[t] ? ld_gather(b + col[u] * ldb + j) : T(0);
          }
        }
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
#pragma unroll
          for (int t = 0; t < J; ++t) acc[t] = add_rn(acc[t], mul_rn(av[u], bv[u][t]));
        }
      }
      for (; q < pe; ++q) {
        const int64_t cq = __ldg(idx + q);
        const T av = mul_rn(alpha, __ldg(val + q));
#pragma unroll
        for (int t = 0; t < J; ++t) {
          const int64_t j = j0 + t * G + lane;
          const T bv = live[t] ? ld_gather(b + cq * ldb + j) : T(0);
          acc[t] = add_rn(acc[t], mul_rn(av, bv));
        }
      }
#pragma unroll
      for (int t = 0; t < J; ++t) {
        const int64_t j = j0 + t * G + lane;
        if (live[t]) c[o * ldc + j] = acc[t];
      }
    }
  }
}

// Row-major B and C with 16-byte aligned rows: each lane owns whole 16-byte
// chunks (4 floats or 2 doubles) of the output row, so one vector load brings
// a chunk of B(c, :) and the arithmetic per column is one multiply-add
// (FAST) or one rounded multiply and one rounded add (EXACT, the reference's
// per-entry update, bit-exact).  G lanes share a row; J chunks per lane.
template <typename T>
struct Chunk;
template <>
struct Chunk<float> {
  using type = float4;
  static constexpr int n = 4;
  __device__ static void split(const float4& v, float (&e)[4]) {
    e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
  }
  __device__ static float4 join(const float (&e)[4]) { return make_float4(e[0], e[1], e[2], e[3]); }
};
template <>
struct Chunk<double> {
  using type = double2;
  static constexpr int n = 2;
  __device__ static void split(const double2& v, double (&e)[2]) {
    e[0] = v.x; e[1] = v.y;
  }
  __device__ static double2 join(const double (&e)[2]) { return make_double2(e[0], e[1]); }
};

template <typename T, int G, int J, bool EXACT>
__global__ void __launch_bounds__(kThreads)
spmm_chunk_kernel(int64_t rows, int64_t chunks, const int64_t* __restrict__ ptr,
                  const int64_t* __restrict__ idx, const T* __restrict__ val,
                  const T* __restrict__ b, int64_t ldb, T* __restrict__ c, int64_t ldc,
                  T alpha) {
  using C = Chunk<T>;
  using V = typename C::type;
  constexpr int N = C::n;
  constexpr int kGroups = kThreads / G;
  const int lane = threadIdx.x % G;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * kGroups + threadIdx.x / G;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kGroups;
  for (int64_t o = first; o < rows; o += step) {
    const int64_t pb = __ldg(ptr + o);
    const int64_t pe = __ldg(ptr + o + 1);
    if (!EXACT && pb == pe) continue;
    T* crow = c + o * ldc;
    for (int64_t v0 = 0; v0 < chunks; v0 += int64_t{G} * J) {
      T acc[J][N];
      bool live[J];
#pragma unroll
      for (int t = 0; t < J; ++t) {
        const int64_t jv = v0 + t * G + lane;
        live[t] = jv < chunks;
        if (EXACT && live[t]) {
          C::split(*reinterpret_cast<const V*>(crow + jv * N), acc[t]);
        } else {
#pragma unroll
          for (int e = 0; e < N; ++e) acc[t][e] = T(0);
        }
      }
      int64_t q = pb;
      for (; q + kEntryUnroll <= pe; q += kEntryUnroll) {
        int64_t col[kEntryUnroll];
        T av[kEntryUnroll];
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
          col[u] = __ldg(idx + q + u);
          av[u] = EXACT ? mul_rn(alpha, __ldg(val + q + u)) : __ldg(val + q + u);
        }
        V bv[kEntryUnroll][J];
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
#pragma unroll
          for (int t = 0; t < J; ++t) {
            const int64_t jv = v0 + t * G + lane;
            bv[u][t] = live[t] ? __ldg(reinterpret_cast<const V*>(b + col[u] * ldb + jv * N))
                               : V{};
          }
        }
#pragma unroll
        for (int u = 0; u < kEntryUnroll; ++u) {
#pragma unroll
          for (int t = 0; t < J; ++t) {
            T e[N];
            C::split(bv[u][t], e);
#pragma unroll
            for (int i = 0; i < N; ++i) {
              acc[t][i] = EXACT ? add_rn(acc[t][i], mul_rn(av[u], e[i]))
                                : fma(av[u], e[i], acc[t][i]);
            }
          }
        }
      }
      for (; q < pe; ++q) {
        const int64_t cq = __ldg(idx + q);
        const T av = EXACT ? mul_rn(alpha, __ldg(val + q)) : __ldg(val + q);
#pragma unroll
        for (int t = 0; t < J; ++t) {
          const int64_t jv = v0 + t * G + lane;
          if (!live[t]) continue;
          T e[N];
          C::split(__ldg(reinterpret_cast<const V*>(b + cq * ldb + jv * N)), e);
#pragma unroll
          for (int i = 0; i < N; ++i) {
            acc[t][i] = EXACT ? add_rn(acc[t][i], mul_rn(av, e[i])) : fma(av, e[i], acc[t][i]);
          }
        }
      }
#pragma unroll
      for (int t = 0; t < J; ++t) {
        const int64_t jv = v0 + t * G + lane;
        if (!live[t]) continue;
        V* cp = reinterpret_cast<V*>(crow + jv * N);
        if (EXACT) {
          *cp = C::join(acc[t]);
        } else {
          T old[N];
          C::split(*cp, old);
#pragma unroll
          for (int i = 0; i < N; ++i) acc[t][i] = fma(alpha, acc[t][i], old[i]);
          *cp = C::join(acc[t]);
        }
      }
    }
  }
}

__device__ __forceinline__ int64_t dense_at(int layout, int64_t ld, int64_t r,
                                            int64_t col) {
  return layout == ASCB_ROW_MAJOR ? r * ld + col : col * ld + r;
}

// Any layout: one thread per output element, entries in stored order.
template <typename T>
__global__ void __launch_bounds__(kThreads)
spmm_general_kernel(int64_t rows, int64_t k, const int64_t* __restrict__ ptr,
                    const int64_t* __restrict__ idx, const T* __restrict__ val,
                    const T* __restrict__ b, int b_layout, int64_t ldb,
                    T* __restrict__ c, int c_layout, int64_t ldc, T alpha) {
  const int64_t count = rows * k;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
       t < count; t += step) {
    // consecutive threads take consecutive elements of C's contiguous axis
    int64_t o, j;
    if (c_layout == ASCB_ROW_MAJOR) {
      o = t / k;
      j = t % k;
    } else {
      j = t / rows;
      o = t % rows;
    }
    T* cp = c + dense_at(c_layout, ldc, o, j);
    T acc = *cp;
    for (int64_t q = __ldg(ptr + o); q < __ldg(ptr + o + 1); ++q) {
      const T av = mul_rn(alpha, __ldg(val + q));
      acc = add_rn(acc, mul_rn(av, ld_gather(b + dense_at(b_layout, ldb, __ldg(idx + q), j))));
    }
    *cp = acc;
  }
}

// Transposed product by scatter: C(c, j) += alpha * v * B(r, j) for every
// stored (r, c, v); one thread per (entry, column).
template <typename T>
__global__ void __launch_bounds__(kThreads)
spmm_scatter_kernel(int64_t rows, int64_t k, const int64_t* __restrict__ ptr,
                    const int64_t* __restrict__ idx, const T* __restrict__ val,
                    const T* __restrict__ b, int b_layout, int64_t ldb,
                    T* __restrict__ c, int c_layout, int64_t ldc, T alpha) {
  // one warp per source row, lanes over (entry, column) pairs
  const int lane = threadIdx.x & 31;
  const int64_t first = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t step = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = first; r < rows; r += step) {
    const int64_t pb = __ldg(ptr + r);
    const int64_t n = (__ldg(ptr + r + 1) - pb) * k;
    for (int64_t t = lane; t < n; t += 32) {
      const int64_t q = pb + t / k;
      const int64_t j = t % k;
      const T term = alpha * __ldg(val + q) * ld_gather(b + dense_at(b_layout, ldb, r, j));
      atomicAdd(c + dense_at(c_layout, ldc, __ldg(idx + q), j), term);
    }
  }
}

unsigned grid_for(int64_t work, int per_block, int sm_count) {
  const int64_t needed = (work + per_block - 1) / per_block;
  const int64_t resident = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
  return static_cast<unsigned>(needed < resident ? (needed > 0 ? needed : 1) : resident);
}

template <typename T, int G, int J>
int launch_rm(cudaStream_t s, const ascb_csr* a, int64_t k, const void* b,
              int64_t ldb, void* c, int64_t ldc, T alpha, int sm) {
  spmm_row_major_kernel<T, G, J><<<grid_for(a->rows, kThreads / G, sm), kThreads, 0, s>>>(
      a->rows, k, a->ptr, a->idx, static_cast<const T*>(a->val),
      static_cast<const T*>(b), ldb, static_cast<T*>(c), ldc, alpha);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, int G, int J>
int launch_chunks(cudaStream_t s, bool exact, const ascb_csr* a, int64_t chunks, const void* b,
                  int64_t ldb, void* c, int64_t ldc, T alpha, int sm) {
  const unsigned grid = grid_for(a->rows, kThreads / G, sm);
  const auto* val = static_cast<const T*>(a->val);
  if (exact) {
    spmm_chunk_kernel<T, G, J, true><<<grid, kThreads, 0, s>>>(
        a->rows, chunks, a->ptr, a->idx, val, static_cast<const T*>(b), ldb,
        static_cast<T*>(c), ldc, alpha);
  } else {
    spmm_chunk_kernel<T, G, J, false><<<grid, kThreads, 0, s>>>(
        a->rows, chunks, a->ptr, a->idx, val, static_cast<const T*>(b), ldb,
        static_cast<T*>(c), ldc, alpha);
  }
  return static_cast<int>(cudaGetLastError());
}

// Chunked kernel choice, measured on B200 with the 27-point stencil and the
// 16 x 16 block-sparse matrices: a row's chunks are spread over G lanes, J
// chunks per lane.  Up to two chunks per row take one lane each (more rows
// per warp); wider rows take two chunks per lane (more independent loads in
// flight, and a CTA covers more consecutive rows whose right-hand-side rows
// then hit in L1).
template <typename T>
int launch_chunked(cudaStream_t s, bool exact, const ascb_csr* a, int64_t chunks,
                   const void* b, int64_t ldb, void* c, int64_t ldc, T alpha, int sm) {
#define ASCB_CHUNKS(G, J) \
  return launch_chunks<T, G, J>(s, exact, a, chunks, b, ldb, c, ldc, alpha, sm)
  if (chunks <= 1) ASCB_CHUNKS(1, 1);
  if (chunks <= 2) ASCB_CHUNKS(2, 1);
  if (chunks <= 4) ASCB_CHUNKS(2, 2);
  if (chunks <= 8) ASCB_CHUNKS(4, 2);
  if (chunks <= 16) ASCB_CHUNKS(8, 2);
  ASCB_CHUNKS(16, 2);
#undef ASCB_CHUNKS
}

template <typename T>
int spmm_typed(cudaStream_t s, int transpose, int exact, const ascb_csr* a, int64_t k,
               const void* b, int b_layout, int64_t ldb, void* c, int c_layout,
               int64_t ldc, double alpha_d, int sm) {
  const T alpha = static_cast<T>(alpha_d);
  if (transpose) {
    spmm_scatter_kernel<T><<<grid_for(a->rows, kThreads / 32, sm), kThreads, 0, s>>>(
        a->rows, k, a->ptr, a->idx, static_cast<const T*>(a->val),
        static_cast<const T*>(b), b_layout, ldb, static_cast<T*>(c), c_layout,
        ldc, alpha);
    return static_cast<int>(cudaGetLastError());
  }
  if (b_layout == ASCB_ROW_MAJOR && c_layout == ASCB_ROW_MAJOR) {
    constexpr int64_t N = Chunk<T>::n;
    const bool chunked = k % N == 0 && ldb % N == 0 && ldc % N == 0 &&
                         ((reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c)) & 15u) == 0;
    // the exact form at 32 or more chunks per row runs faster on the scalar
    // kernel below (measured on both matrices above)
    if (chunked && !(exact && k / N >= 32)) {
      return launch_chunked<T>(s, exact != 0, a, k / N, b, ldb, c, ldc, alpha, sm);
    }
    if (k <= 8) return launch_rm<T, 8, 1>(s, a, k, b, ldb, c, ldc, alpha, sm);
    if (k <= 16) return launch_rm<T, 16, 1>(s, a, k, b, ldb, c, ldc, alpha, sm);
    if (k <= 32) return launch_rm<T, 32, 1>(s, a, k, b, ldb, c, ldc, alpha, sm);
    if (k <= 64) return launch_rm<T, 32, 2>(s, a, k, b, ldb, c, ldc, alpha, sm);
    return launch_rm<T, 32, 4>(s, a, k, b, ldb, c, ldc, alpha, sm);
  }
  spmm_general_kernel<T><<<grid_for(a->rows * k, kThreads, sm), kThreads, 0, s>>>(
      a->rows, k, a->ptr, a->idx, static_cast<const T*>(a->val),
      static_cast<const T*>(b), b_layout, ldb, static_cast<T*>(c), c_layout,
      ldc, alpha);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, int LANES>
__global__ void __launch_bounds__(kThreads)
spmv_scatter_kernel(int64_t rows, const int64_t* __restrict__ ptr,
                    const int64_t* __restrict__ idx, const T* __restrict__ val,
                    const T* __restrict__ x, int64_t incx, T* __restrict__ y,
                    int64_t incy, T alpha) {
  constexpr int kGroups = kThreads / LANES;
  const int lane = threadIdx.x % LANES;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * kGroups + threadIdx.x / LANES;
  const int64_t step = static_cast<int64_t>(gridDim.x) * kGroups;
  for (int64_t r = first; r < rows; r += step) {
    const T ax = alpha * ld_gather(x + r * incx);
    for (int64_t q = __ldg(ptr + r) + lane; q < __ldg(ptr + r + 1); q += LANES) {
      atomicAdd(y + ld_stream(idx + q) * incy, ld_stream(val + q) * ax);
    }
  }
}

}  // namespace
}  // namespace ascb

extern "C" {

int ascb_spmm(void* stream, int dtype, int transpose, int exact, const ascb_csr* a,
              int64_t k, const void* b, int b_layout, int64_t ldb, void* c,
              int c_layout, int64_t ldc, double alpha, int sm_count) {
  if (a->rows <= 0 || k <= 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == ASCB_F64
             ? ascb::spmm_typed<double>(s, transpose, exact, a, k, b, b_layout, ldb, c,
                                        c_layout, ldc, alpha, sm_count)
             : ascb::spmm_typed<float>(s, transpose, exact, a, k, b, b_layout, ldb, c,
                                       c_layout, ldc, alpha, sm_count);
}

int ascb_spmv_scatter(void* stream, int dtype, const ascb_csr* a, double alpha,
                      const ascb_vec* x, const ascb_vec* y, int sm_count) {
  if (a->rows <= 0 || a->nnz == 0) return 0;
  auto s = static_cast<cudaStream_t>(stream);
  const unsigned blocks = ascb::grid_for(a->rows, ascb::kThreads / 8, sm_count);
  if (dtype == ASCB_F64) {
    ascb::spmv_scatter_kernel<double, 8><<<blocks, ascb::kThreads, 0, s>>>(
        a->rows, a->ptr, a->idx, static_cast<const double*>(a->val),
        static_cast<const double*>(x->data), x->stride,
        static_cast<double*>(y->data), y->stride, alpha);
  } else {
    ascb::spmv_scatter_kernel<float, 8><<<blocks, ascb::kThreads, 0, s>>>(
        a->rows, a->ptr, a->idx, static_cast<const float*>(a->val),
        static_cast<const float*>(x->data), x->stride,
        static_cast<float*>(y->data), y->stride, static_cast<float>(alpha));
  }
  return static_cast<int>(cudaGetLastError());
}

}  // extern "C"
