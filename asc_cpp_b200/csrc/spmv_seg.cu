// Register-segmented CSR SpMV for sm_100a (the default SpMV kernel, both
// numerical modes).
//
// Row tiles: tile k holds the rows r with W*r + ptr[r] in [I*k, I*(k+1)):
// the warp tiles (W = 8, I = 256: at most 32 rows) or the kernel's own tiles
// (W = 2, I = 251: at most 125 rows, so short rows leave less of each window
// empty).  For one tile:
//   * the window -- at most 256 nonzero positions from the aligned position
//     at or before the tile's first nonzero -- is split into 32 lanes x 8
//     CONTIGUOUS positions; each lane fetches its column indices and values
//     with 16- or 32-byte vector loads straight into registers (every sector
//     touched once with 32-byte loads) and keeps 8 x gathers in flight;
//   * FAST: a 256-bit shared bitmap marks the positions where rows start,
//     each lane runs a segmented sum over its 8 products, and one segmented
//     warp scan joins the rows that cross lanes;
//     |y - y_ref| <= gamma_{n+2}(|alpha||A||x| + |beta||y|);
//   * EXACT: the products are formed in parallel and kept in shared memory,
//     then lane k adds the products of the tile's rows k, k + 32, ... in
//     stored order -- every row is summed exactly as the serial reference
//     does, all rows of the tile at once.
// Every row of a tile but the last ends inside its window; the last may run
// on, and its remainder is reduced by the whole warp in rounds of 256
// (EXACT: added in stored order by its lane; ROW_SPLIT: long tails handed to
// a second kernel).
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kThreads = kWarpsPerCta * 32;
constexpr int kItems = 256;        // weighted items per tile (= positions)
constexpr int kRowWeight = kItems / 32;  // the warp-tile partition: at most 32 rows
// Row weight of the segmented kernel's own partition (ascb_seg_tile_row_weight):
// a tile holds at most kItems / weight rows, so a smaller weight leaves more of
// each 256-position window to nonzeros on matrices with short rows.
#ifndef ASCB_SEG_ROW_WEIGHT
#define ASCB_SEG_ROW_WEIGHT 2
#endif
constexpr int kSegWeight = ASCB_SEG_ROW_WEIGHT;
constexpr int kMaxRowsPerLane = kRowWeight / kSegWeight;  // rows per lane in a tile
static_assert(kRowWeight % kSegWeight == 0 && kMaxRowsPerLane >= 1 && kMaxRowsPerLane <= 8,
              "the segmented kernel's row weight divides 8");
// A window starts on the aligned position at or before its tile's first
// nonzero, up to kMaxLead positions earlier (FP32 with 32-byte loads).  Every
// row of a tile but the first must start inside the window, so a tile of row
// weight W spans at most tile_items<RPL>() weighted items: its other rows then
// start at most items - 1 - W <= kItems - 1 - kMaxLead positions past its
// first row's start (the warp tiles' W = 8 needs no reduction).
constexpr int kMaxLead = 7;
template <int RPL>
__host__ __device__ constexpr int64_t tile_items() {
  return kRowWeight / RPL >= kMaxLead ? kItems : kItems - kMaxLead + kRowWeight / RPL;
}
constexpr int kPer = 8;            // contiguous positions per lane
constexpr int kChunk = 32;         // tile bounds cached per warp
constexpr int kMaxDevices = 64;
// CTAs per SM the segmented kernels are compiled for (register cap): on the
// 4M-row power-law matrix (B200) the contracted tile runs best at 7 (72
// registers: 2621 / 2667 GB/s plain / row split, against 2567 / 2524 at 6),
// the bit-exact tile at 6 (2250 against 2168 GB/s at 7, and 1895 at 5).
constexpr int kMinCtasFast = 7;
constexpr int kMinCtasExact = 6;

// Row split (BACKEND_DEFAULT): a tile whose last row runs more than
// `split_min` positions past the tile's window does not walk that tail
// itself.  It reserves an entry {row, first tail position, end, first chunk}
// and stores the row's sum up to the window end as the entry's head; the
// split kernel's warps then take the tail in 256-position chunks, each
// writing one partial, and the warp that completes an entry's last chunk adds
// head + partials in chunk order (a fixed tree), so results repeat run to run.
struct SplitEntry {
  int64_t row;    // < 0: not split (over capacity; never the case within bounds)
  int64_t start;  // first tail position (16-byte aligned: the window end)
  int64_t end;    // one past the row's last position
  int64_t chunk;  // first chunk of this entry
};
struct SplitBlock {
  unsigned long long* packed;  // (entries << 40) | chunks reserved; zero at launch
  int* done;                   // chunks finished per entry; zero at launch
  SplitEntry* entries;
  void* head;                  // per entry, T
  void* partial;               // per chunk, T
  int64_t max_entries;
  int64_t max_chunks;
  int64_t split_min;
};
constexpr unsigned long long kChunkMask = (1ull << 40) - 1;

template <typename T>
struct SegSmem {
  uint32_t bits[kItems / 32 + 1];  // row-start bitmap of positions 0..256
  int16_t rowid[32 * 8 + 1];       // k-th nonempty row of the tile -> its offset (RPL <= 8)
  int64_t bnd[kChunk + 1];         // first row of tiles c0 .. c0 + kChunk
  alignas(16) T prod[kItems];      // exact form: the window's / a long row's products
};

// Arithmetic of the two modes.  EXACT rounds every product and sum separately
// in the reference's order: compat s = +0 + v*x + ..., y = alpha*s + beta*y
// (src/sparse/reference_blas.cc:13-39); standard s = y + (alpha*v)*x + ...
// (include/asc/sparse/blas.h:1653-1665).  FAST forms plain sums.
template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T product(T alpha, T v, T xv) {
  if (EXACT && STANDARD) return mul_rn(mul_rn(alpha, v), xv);
  return EXACT ? mul_rn(v, xv) : v * xv;
}
template <bool EXACT, typename T>
__device__ __forceinline__ T add(T a, T b) {
  return EXACT ? add_rn(a, b) : a + b;
}
template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T row_init(T y_old) {
  return (EXACT && STANDARD) ? y_old : T(0);
}

template <typename T>
__device__ __forceinline__ void load_vec2(const T* p, T& a, T& b);
template <>
__device__ __forceinline__ void load_vec2<double>(const double* p, double& a, double& b) {
  const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
  a = v.x;
  b = v.y;
}
__device__ __forceinline__ void load_idx2(const int64_t* p, int64_t& a, int64_t& b) {
  const longlong2 v = __ldcs(reinterpret_cast<const longlong2*>(p));
  a = v.x;
  b = v.y;
}

template <bool EXACT, bool STANDARD, typename T>
__device__ __forceinline__ T finish(T s, T alpha, T beta, const T* yp) {
  if (EXACT) {
    if (STANDARD) return s;
    T r = mul_rn(alpha, s);
    if (beta != T(0)) r = add_rn(r, mul_rn(beta, *yp));
    return r;
  }
  if (STANDARD) return fma(alpha, s, *yp);
  return beta != T(0) ? fma(alpha, s, beta * *yp) : alpha * s;
}

// Products of the lane's 8 positions, read from ip[0..8) / vp[0..8) (16-byte
// aligned); bit k of vmask says whether position k holds a nonzero of the
// window.  Invalid positions give 0.  16-byte chunks that are wholly valid are
// fetched with one vector load, others element by element.
template <typename T, bool EXACT, bool STANDARD, bool UNIT, bool V32 = false>
__device__ __forceinline__ void lane_products(T (&p)[kPer], uint32_t vmask,
                                              const int64_t* __restrict__ ip,
                                              const T* __restrict__ vp, const T* __restrict__ x,
                                              int64_t incx, T alpha) {
  int64_t c[kPer];
  T v[kPer];
  if constexpr (V32) {
    // 32-byte aligned: one request per 32 bytes, so each sector a lane reads
    // is touched once (16-byte loads touch every sector of a lane's run twice)
#pragma unroll
    for (int k = 0; k < kPer; k += 4) {
      if (((vmask >> k) & 15u) == 15u) {
        ld_stream32(ip + k, c + k);
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) c[k + u] = ((vmask >> (k + u)) & 1u) ? ld_stream(ip + k + u) : 0;
      }
    }
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int k = 0; k < kPer; k += 4) {
        if (((vmask >> k) & 15u) == 15u) {
          ld_stream32(vp + k, v + k);
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            v[k + u] = ((vmask >> (k + u)) & 1u) ? ld_stream(vp + k + u) : T(0);
          }
        }
      }
    } else {
      if (vmask == 0xffu) {
        ld_stream32(vp, v);
      } else {
#pragma unroll
        for (int u = 0; u < kPer; ++u) v[u] = ((vmask >> u) & 1u) ? ld_stream(vp + u) : T(0);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < kPer; k += 2) {
      if (((vmask >> k) & 3u) == 3u) {
        load_idx2(ip + k, c[k], c[k + 1]);
      } else {
        c[k] = ((vmask >> k) & 1u) ? ld_stream(ip + k) : 0;
        c[k + 1] = ((vmask >> (k + 1)) & 1u) ? ld_stream(ip + k + 1) : 0;
      }
    }
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int k = 0; k < kPer; k += 2) {
        if (((vmask >> k) & 3u) == 3u) {
          load_vec2(vp + k, v[k], v[k + 1]);
        } else {
          v[k] = ((vmask >> k) & 1u) ? ld_stream(vp + k) : T(0);
          v[k + 1] = ((vmask >> (k + 1)) & 1u) ? ld_stream(vp + k + 1) : T(0);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < kPer; k += 4) {
        if (((vmask >> k) & 15u) == 15u) {
          const float4 f = __ldcs(reinterpret_cast<const float4*>(vp + k));
          v[k] = f.x;
          v[k + 1] = f.y;
          v[k + 2] = f.z;
          v[k + 3] = f.w;
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            v[k + u] = ((vmask >> (k + u)) & 1u) ? ld_stream(vp + k + u) : T(0);
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    p[k] = ((vmask >> k) & 1u)
               ? product<EXACT, STANDARD>(alpha, v[k], ld_gather(&at<UNIT>(x, c[k], incx)))
               : T(0);
  }
}

// A lane's 8 products into its 8 consecutive shared-memory slots.  Lane l
// owns bytes [8 l sizeof(T), ...): stored chunk by chunk in the same order by
// every lane, every second (FP64) or fourth (FP32) lane hits the same banks.
// FP64: lane l stores its 16-byte chunk j ^ ((l / 2) & 1) in step j, so each
// 16-byte store meets at most 2-way conflicts for 16 selects per lane (the
// conflict-free rotation (j + l / 2) % 4 needs 48 and measured 2.3% slower on
// the 4M-row power-law matrix).  FP32: chunk (j + l / 4) % 2, conflict-free.
__device__ __forceinline__ void store_run(double* dst, int lane, const double (&p)[kPer]) {
  const bool h = ((lane >> 1) & 1) != 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = j ^ (h ? 1 : 0);
    double2 v;
    v.x = h ? p[2 * (j ^ 1)] : p[2 * j];
    v.y = h ? p[2 * (j ^ 1) + 1] : p[2 * j + 1];
    *reinterpret_cast<double2*>(dst + 2 * c) = v;
  }
}
__device__ __forceinline__ void store_run(float* dst, int lane, const float (&p)[kPer]) {
  const bool h = ((lane >> 2) & 1) != 0;
  const float4 lo = make_float4(p[0], p[1], p[2], p[3]);
  const float4 hi = make_float4(p[4], p[5], p[6], p[7]);
  *reinterpret_cast<float4*>(dst + (h ? 4 : 0)) = h ? hi : lo;
  *reinterpret_cast<float4*>(dst + (h ? 0 : 4)) = h ? lo : hi;
}

// acc + prod[q] + prod[q + 1] + ... + prod[e - 1], each sum rounded, in that
// order; the aligned middle is read with 16-byte shared loads (prod is
// 16-byte aligned).
__device__ __forceinline__ double chain_sum(double acc, const double* prod, int q, int e) {
  if ((q & 1) && q < e) acc = add_rn(acc, prod[q++]);
  for (; q + 4 <= e; q += 4) {
    const double2 u = *reinterpret_cast<const double2*>(prod + q);
    const double2 v = *reinterpret_cast<const double2*>(prod + q + 2);
    acc = add_rn(add_rn(add_rn(add_rn(acc, u.x), u.y), v.x), v.y);
  }
  if (q + 2 <= e) {
    const double2 u = *reinterpret_cast<const double2*>(prod + q);
    acc = add_rn(add_rn(acc, u.x), u.y);
    q += 2;
  }
  if (q < e) acc = add_rn(acc, prod[q]);
  return acc;
}
__device__ __forceinline__ float chain_sum(float acc, const float* prod, int q, int e) {
  for (; (q & 3) && q < e; ++q) acc = add_rn(acc, prod[q]);
  for (; q + 4 <= e; q += 4) {
    const float4 u = *reinterpret_cast<const float4*>(prod + q);
    acc = add_rn(add_rn(add_rn(add_rn(acc, u.x), u.y), u.z), u.w);
  }
  for (; q < e; ++q) acc = add_rn(acc, prod[q]);
  return acc;
}

// EXACT tile: the window's products are formed in parallel (8 contiguous
// positions per lane, as in the contracted tile) and staged in shared memory;
// then lane k, which holds row r0 + k's bounds, adds that row's products in
// stored order from shared memory -- the serial reference's chain, with every
// row of the tile summed at once by its own lane.  A last row that runs past
// the window continues in rounds of 256 products (all lanes form them, its
// lane adds them).  No per-position bitmap, ranks or lane-to-lane hand-over:
// the instruction count per tile follows the longest row, not the number of
// lane boundaries the rows cross.
template <typename T, bool STANDARD, bool UNIT, bool V32, int RPL>
__device__ __forceinline__ void exact_tile(SegSmem<T>& w, int lane,
                                           const int64_t* __restrict__ ptr,
                                           const int64_t* __restrict__ idx,
                                           const T* __restrict__ val, const T* __restrict__ x,
                                           int64_t incx, T* __restrict__ y, int64_t incy,
                                           T alpha, T beta, int64_t r0, int nr, int64_t rb,
                                           int64_t re) {
  constexpr int64_t kAlign = V32 ? (sizeof(T) == 8 ? 4 : 8) : (sizeof(T) == 8 ? 2 : 4);
  const int64_t base = __shfl_sync(0xffffffffu, rb, 0);
  const int64_t span =
      (nr <= 32 ? __shfl_sync(0xffffffffu, re, nr - 1) : __ldg(ptr + r0 + nr)) - base;
  const int64_t a0 = base / kAlign * kAlign;
  const int lo = static_cast<int>(base - a0);
  const int window = static_cast<int>(span < kItems - lo ? span : kItems - lo);
  const int lim = lo + window;
  const bool ends_here = span <= window;

  const int p0 = kPer * lane;
  const int vlo = lo - p0 < 0 ? 0 : (lo - p0 > kPer ? kPer : lo - p0);
  const int vhi = lim - p0 < 0 ? 0 : (lim - p0 > kPer ? kPer : lim - p0);
  const uint32_t vmask = ((1u << vhi) - 1u) & ~((1u << vlo) - 1u);
  T p[kPer];
  lane_products<T, true, STANDARD, UNIT, V32>(p, vmask, idx + (a0 + p0), val + (a0 + p0), x, incx,
                                              alpha);
  store_run(w.prod + p0, lane, p);
  __syncwarp();

  // lane l sums rows l, l + 32, ... (tiles of more than 32 rows: the bounds of
  // rows past the first 32 are read here)
  const bool carries = !ends_here && lane == (nr - 1) % 32;  // owns the row that runs on
  T acc = T(0);
  T* yp = nullptr;
#pragma unroll
  for (int m = 0; m < RPL; ++m) {
    if (32 * m >= nr) break;
    const int k = lane + 32 * m;
    if (k >= nr) continue;
    const int64_t b = m == 0 ? rb : __ldg(ptr + r0 + k);
    const int64_t e = m == 0 ? re : __ldg(ptr + r0 + k + 1);
    T* rp = &at<UNIT>(y, r0 + k, incy);
    T racc = STANDARD ? *rp : T(0);
    const int s0 = static_cast<int>(b - a0);
    const int e0 = static_cast<int>(e - a0 < lim ? e - a0 : lim);
    racc = chain_sum(racc, w.prod, s0, e0);
    if (carries && k == nr - 1) {
      acc = racc;
      yp = rp;
    } else {
      *rp = finish<true, STANDARD>(racc, alpha, beta, rp);
    }
  }
  if (!ends_here) {
    // the last row past the window: rounds of 256 products, added in stored
    // order by its lane (the window ends on an aligned position, a0 + 256)
    for (int64_t q0 = base + window; q0 < base + span; q0 += kItems) {
      const int64_t rem = base + span - q0;
      const int cnt = static_cast<int>(rem < kItems ? rem : kItems);
      const int hi = cnt - p0 < 0 ? 0 : (cnt - p0 > kPer ? kPer : cnt - p0);
      T q[kPer];
      __syncwarp();  // the previous round's products have been read
      lane_products<T, true, STANDARD, UNIT, V32>(q, (1u << hi) - 1u, idx + (q0 + p0),
                                                  val + (q0 + p0), x, incx, alpha);
      store_run(w.prod + p0, lane, q);
      __syncwarp();
      if (carries) acc = chain_sum(acc, w.prod, 0, cnt);
    }
    if (carries) *yp = finish<true, STANDARD>(acc, alpha, beta, yp);
  }
  __syncwarp();  // the product buffer is rewritten by the next tile
}

// One tile: rows r0 .. r0 + nr - 1 (nr >= 1), whose ptr entries lane k holds
// as rb = ptr[r0 + k], re = ptr[r0 + k + 1] (k < nr).  Shared by the
// single-matrix and the batched kernels.
template <typename T, bool EXACT, bool STANDARD, bool UNIT, bool SPLIT = false, bool V32 = false,
          int RPL = 1>
__device__ __forceinline__ void seg_tile(SegSmem<T>& w, int lane, const int64_t* __restrict__ ptr,
                                         const int64_t* __restrict__ idx,
                                         const T* __restrict__ val, const T* __restrict__ x,
                                         int64_t incx, T* __restrict__ y, int64_t incy, T alpha,
                                         T beta, int64_t r0, int nr, int64_t rb, int64_t re,
                                         const SplitBlock* split = nullptr) {
  if constexpr (EXACT) {
    exact_tile<T, STANDARD, UNIT, V32, RPL>(w, lane, ptr, idx, val, x, incx, y, incy, alpha, beta,
                                            r0, nr, rb, re);
    return;
  }
  const unsigned lt_mask = (1u << lane) - 1u;
  // window start alignment: each lane's 8 values and 8 indices start on a
  // 16-byte (V32: 32-byte) boundary (the arrays are aligned so, checked by
  // the host)
  constexpr int64_t kAlign = V32 ? (sizeof(T) == 8 ? 4 : 8) : (sizeof(T) == 8 ? 2 : 4);

  const int64_t base = __shfl_sync(0xffffffffu, rb, 0);
  const int64_t span =
      (nr <= 32 ? __shfl_sync(0xffffffffu, re, nr - 1) : __ldg(ptr + r0 + nr)) - base;
  const int64_t a0 = base / kAlign * kAlign;
  const int lo = static_cast<int>(base - a0);
  const int window = static_cast<int>(span < kItems - lo ? span : kItems - lo);
  const int lim = lo + window;
  const bool ends_here = span <= window;  // the last row ends in the window

  // row-start bitmap (+ end marker at lim) and nonempty-row table; lane l
  // handles rows l, l + 32, ... (bounds past the first 32 rows read here)
  if (lane <= kItems / 32) w.bits[lane] = 0u;
  __syncwarp();
  int ne_before = 0;  // nonempty rows in earlier passes
#pragma unroll
  for (int m = 0; m < RPL; ++m) {
    if (32 * m >= nr) break;
    const int k = lane + 32 * m;
    const bool mine = k < nr;
    const int64_t b = m == 0 ? rb : (mine ? __ldg(ptr + r0 + k) : 0);
    const int64_t e = m == 0 ? re : (mine ? __ldg(ptr + r0 + k + 1) : 0);
    const bool nonempty = mine && e > b;
    if (nonempty) {
      const int sp = static_cast<int>(b - a0);
      atomicOr(&w.bits[sp >> 5], 1u << (sp & 31));
    }
    const unsigned ne_mask = __ballot_sync(0xffffffffu, nonempty);
    if (nonempty) w.rowid[ne_before + __popc(ne_mask & lt_mask)] = static_cast<int16_t>(k);
    if (mine && !nonempty && !STANDARD) {  // empty row: y = alpha*(+0) + beta*y
      T* yp = &at<UNIT>(y, r0 + k, incy);
      *yp = finish<EXACT, STANDARD>(T(0), alpha, beta, yp);
    }
    ne_before += __popc(ne_mask);
  }
  if (lane == 0 && ends_here) atomicOr(&w.bits[lim >> 5], 1u << (lim & 31));
  __syncwarp();

  // lane's 8 contiguous positions [8*lane, 8*lane + 8) of the window
  const int p0 = kPer * lane;
  const int vlo = lo - p0 < 0 ? 0 : (lo - p0 > kPer ? kPer : lo - p0);
  const int vhi = lim - p0 < 0 ? 0 : (lim - p0 > kPer ? kPer : lim - p0);
  const uint32_t vmask = ((1u << vhi) - 1u) & ~((1u << vlo) - 1u);
  T p[kPer];
  lane_products<T, EXACT, STANDARD, UNIT, V32>(p, vmask, idx + (a0 + p0), val + (a0 + p0), x, incx,
                                          alpha);
  const uint32_t word = w.bits[lane >> 2];
  const uint32_t flags = (word >> ((lane & 3) * 8)) & 0xffu;
  const uint32_t next_word = w.bits[(lane + 1) >> 2];
  const bool next_start = ((next_word >> (((lane + 1) & 3) * 8)) & 1u) != 0u;
  // segment ranks: starts strictly before this lane
  int before = __popc(flags);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, before, o);
    if (lane >= o) before += v;
  }
  before -= __popc(flags);  // exclusive

  // local segmented sum.  A segment that starts inside the lane is summed
  // here (in stored order); the lane's first segment, when it continues a
  // row from earlier lanes, is joined below.
  const bool has_data = vmask != 0u;
  int rank = before;  // rows started at or before the current position
  T acc = T(0);
  bool first_seg = true;  // still in the segment open at the lane's start
  T first_val = T(0);
  int first_rank = -1;
  int first_end = kPer;   // position where the continued segment closes
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    if ((flags >> i) & 1u) {
      if (i > 0 && p0 + i > lo) {  // close the segment before position i
        if (first_seg) {
          first_val = acc;
          first_rank = rank;
          first_end = i;
        } else {
          T* yp = &at<UNIT>(y, r0 + w.rowid[rank - 1], incy);
          *yp = finish<EXACT, STANDARD>(acc, alpha, beta, yp);
        }
      }
      first_seg = false;
      ++rank;
      acc = p[i];
    } else if (!(EXACT && first_seg)) {
      acc = add<EXACT>(acc, p[i]);
    }
  }
  const bool has_start = flags != 0u;
  T c;  // this lane's carry out: the running sum of the row open at its end
  T carry_in = T(0);
  if (!EXACT) {
    // segmented scan of the open tails: c = has_start ? acc : c_prev + acc
    c = acc;
    bool f = has_start;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T cu = __shfl_up_sync(0xffffffffu, c, o);
      const bool fu = __shfl_up_sync(0xffffffffu, f, o);
      if (lane >= o) {
        if (!f) c = cu + c;
        f = f || fu;
      }
    }
    carry_in = __shfl_up_sync(0xffffffffu, c, 1);
    if (lane == 0) carry_in = T(0);
    if (first_rank > 0) {  // continued row closed inside this lane
      T* yp = &at<UNIT>(y, r0 + w.rowid[first_rank - 1], incy);
      *yp = finish<EXACT, STANDARD>(carry_in + first_val, alpha, beta, yp);
    }
  } else {
    // exact: the running sum is handed lane to lane; a lane whose first
    // valid position starts a row (or that has no data) needs nothing.
    bool resolved = !has_data || ((flags >> vlo) & 1u);
    c = acc;
    for (int step = 0; step < 32; ++step) {
      const T cu = __shfl_up_sync(0xffffffffu, c, 1);
      const bool ru = __shfl_up_sync(0xffffffffu, resolved, 1);
      if (!resolved && ru) {
        T s = cu;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
          if (k >= vlo && k < first_end) s = add_rn(s, p[k]);
        }
        if (first_rank > 0) {
          T* yp = &at<UNIT>(y, r0 + w.rowid[first_rank - 1], incy);
          *yp = finish<EXACT, STANDARD>(s, alpha, beta, yp);
          c = acc;
        } else {
          c = s;
        }
        resolved = true;
      }
      if (__all_sync(0xffffffffu, resolved)) break;
    }
  }
  if (has_data && next_start && rank > 0 && p0 + kPer <= lim) {
    // the open segment closes at the lane end (row start or data end next)
    T* yp = &at<UNIT>(y, r0 + w.rowid[rank - 1], incy);
    *yp = finish<EXACT, STANDARD>(c, alpha, beta, yp);
  }
  const T carry_out = __shfl_sync(0xffffffffu, c, 31);

  if constexpr (SPLIT) {
    if (!ends_here && span - window > split->split_min) {
      // hand the tail to the split kernel: reserve an entry and its chunks
      int64_t e = -1;
      if (lane == 0) {
        const int64_t tail = span - window;
        const unsigned long long chunks =
            static_cast<unsigned long long>((tail + kItems - 1) / kItems);
        const unsigned long long old = atomicAdd(split->packed, (1ull << 40) | chunks);
        const int64_t entry = static_cast<int64_t>(old >> 40);
        const int64_t first = static_cast<int64_t>(old & kChunkMask);
        if (entry < split->max_entries) {
          const bool fits = first + static_cast<int64_t>(chunks) <= split->max_chunks;
          split->entries[entry] = {fits ? r0 + nr - 1 : -1, base + window, base + span, first};
          static_cast<T*>(split->head)[entry] = carry_out;
          if (fits) e = entry;
        }
      }
      e = __shfl_sync(0xffffffffu, e, 0);
      if (e >= 0) {
        __syncwarp();
        return;
      }
    }
  }
  if (!ends_here) {
    // long last row: the nonzeros past the window, 256 per round, each lane
    // 8 contiguous ones with vector loads (the window ends on an aligned
    // position: a0 + kItems, so every round starts aligned too)
    T total;
    T part = T(0);
    total = carry_out;
    for (int64_t q0 = base + window; q0 < base + span; q0 += kItems) {
      const int64_t rem = base + span - q0;
      const int cnt = static_cast<int>(rem < kItems ? rem : kItems);
      const int hi = cnt - p0 < 0 ? 0 : (cnt - p0 > kPer ? kPer : cnt - p0);
      const uint32_t m = (1u << hi) - 1u;
      T q[kPer];
      lane_products<T, EXACT, STANDARD, UNIT, V32>(q, m, idx + (q0 + p0), val + (q0 + p0), x, incx,
                                              alpha);
      if (!EXACT) {
#pragma unroll
        for (int k = 0; k < kPer; ++k) part += q[k];
      } else {
        // stored order: lane 0 adds the round's products from shared memory
        store_run(w.prod + p0, lane, q);
        __syncwarp();
        if (lane == 0) {
          int k = 0;
          for (; k + 8 <= cnt; k += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) total = add_rn(total, w.prod[k + u]);
          }
          for (; k < cnt; ++k) total = add_rn(total, w.prod[k]);
        }
        __syncwarp();
      }
    }
    if (!EXACT) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += shfl_xor(part, o);
      total = carry_out + part;
    }
    if (lane == 0) {
      T* yp = &at<UNIT>(y, r0 + nr - 1, incy);
      *yp = finish<EXACT, STANDARD>(total, alpha, beta, yp);
    }
  }
  __syncwarp();  // bitmap and row tables are rewritten by the next tile
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT, bool SPLIT = false, bool V32 = false,
          int RPL = 1>
__global__ void __launch_bounds__(kThreads, EXACT ? kMinCtasExact : kMinCtasFast)
seg_kernel(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
           const T* __restrict__ val, const T* __restrict__ x, int64_t incx, T* __restrict__ y,
           int64_t incy, T alpha, T beta, const int64_t* __restrict__ tile_row, int64_t ntiles,
           int64_t rows, int64_t nnz, SplitBlock split) {
  __shared__ SegSmem<T> smem_all[kWarpsPerCta];
  const int lane = threadIdx.x & 31;
  SegSmem<T>& w = smem_all[threadIdx.x >> 5];

  const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + (threadIdx.x >> 5);
  const int64_t warp_count = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  const int64_t per_warp = (ntiles + warp_count - 1) / warp_count;
  const int64_t tb = warp_id * per_warp;
  const int64_t te = tb + per_warp < ntiles ? tb + per_warp : ntiles;
  if (tb >= te) return;

  int64_t c0 = -2 * kChunk;
  auto tile_bounds = [&](int64_t u, int64_t& r0, int& nr) {
    if (u + 1 > c0 + kChunk) {
      __syncwarp();
      c0 = u;
      for (int i = lane; i <= kChunk; i += 32) {
        const int64_t v = c0 + i;
        int64_t b = rows;
        if (v < ntiles) {
          b = tile_row != nullptr ? __ldg(tile_row + v)
                                  : first_row_at(ptr, rows, kRowWeight / RPL, v * tile_items<RPL>());
        }
        w.bnd[i] = b;
      }
      __syncwarp();
    }
    r0 = w.bnd[u - c0];
    nr = static_cast<int>(w.bnd[u - c0 + 1] - r0);
  };

  // prefetch of the next tile's row bounds (one round trip ahead)
  int64_t r0_n;
  int nr_n;
  tile_bounds(tb, r0_n, nr_n);
  int64_t rb_n = lane < nr_n ? __ldg(ptr + r0_n + lane) : 0;
  int64_t re_n = lane < nr_n ? __ldg(ptr + r0_n + lane + 1) : 0;

  for (int64_t t = tb; t < te; ++t) {
    const int64_t r0 = r0_n;
    const int nr = nr_n;
    const int64_t rb = rb_n;
    const int64_t re = re_n;
    if (t + 1 < te) {
      tile_bounds(t + 1, r0_n, nr_n);
      rb_n = lane < nr_n ? __ldg(ptr + r0_n + lane) : 0;
      re_n = lane < nr_n ? __ldg(ptr + r0_n + lane + 1) : 0;
    }
    if (nr == 0) continue;
    seg_tile<T, EXACT, STANDARD, UNIT, SPLIT, V32, RPL>(w, lane, ptr, idx, val, x, incx, y, incy,
                                                       alpha, beta, r0, nr, rb, re, &split);
  }
  (void)nnz;
}

// Tails of the split rows: warp-strided over the reserved chunks.  Chunk c of
// entry e covers positions [start + 256 (c - chunk), ...) of its row; the
// warp that finishes an entry's last chunk writes y.
template <typename T, bool STANDARD, bool UNIT, bool V32>
__global__ void __launch_bounds__(kThreads)
split_chunk_kernel(const int64_t* __restrict__ idx, const T* __restrict__ val,
                   const T* __restrict__ x, int64_t incx, T* __restrict__ y, int64_t incy,
                   T alpha, T beta, SplitBlock split) {
  const int lane = threadIdx.x & 31;
  const unsigned long long packed = __ldcg(split.packed);
  const int64_t entries = min(static_cast<int64_t>(packed >> 40), split.max_entries);
  const int64_t chunks = min(static_cast<int64_t>(packed & kChunkMask), split.max_chunks);
  const int64_t warp_id = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + (threadIdx.x >> 5);
  const int64_t warp_count = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  const T* head = static_cast<const T*>(split.head);
  T* partial = static_cast<T*>(split.partial);
  const int p0 = kPer * lane;
  for (int64_t c = warp_id; c < chunks; c += warp_count) {
    // entry of chunk c: the last one whose first chunk is <= c (entries are
    // reserved in increasing chunk order)
    int64_t lo = 0, hi = entries - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (__ldcg(&split.entries[mid].chunk) <= c) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    const int64_t row = __ldcg(&split.entries[lo].row);
    if (row < 0) continue;
    const int64_t start = __ldcg(&split.entries[lo].start);
    const int64_t end = __ldcg(&split.entries[lo].end);
    const int64_t first = __ldcg(&split.entries[lo].chunk);
    const int64_t n_chunks = (end - start + kItems - 1) / kItems;
    const int64_t q0 = start + (c - first) * kItems;
    const int64_t rem = end - q0;
    const int cnt = static_cast<int>(rem < kItems ? rem : kItems);
    const int hiv = cnt - p0 < 0 ? 0 : (cnt - p0 > kPer ? kPer : cnt - p0);
    T q[kPer];
    lane_products<T, false, STANDARD, UNIT, V32>(q, (1u << hiv) - 1u, idx + (q0 + p0),
                                                 val + (q0 + p0), x, incx, alpha);
    T part = T(0);
#pragma unroll
    for (int k = 0; k < kPer; ++k) part += q[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += shfl_xor(part, o);
    int finished = 0;
    if (lane == 0) {
      partial[c] = part;
      __threadfence();
      finished = atomicAdd(split.done + lo, 1) == n_chunks - 1;
    }
    finished = __shfl_sync(0xffffffffu, finished, 0);
    if (finished) {
      __threadfence();
      // head + partials in a fixed order: lane l adds chunks l, l + 32, ...
      T s = T(0);
      for (int64_t j = lane; j < n_chunks; j += 32) s += __ldcg(partial + first + j);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += shfl_xor(s, o);
      if (lane == 0) {
        T* yp = &at<UNIT>(y, row, incy);
        *yp = finish<false, STANDARD>(__ldcg(head + lo) + s, alpha, beta, yp);
      }
    }
  }
}

// ---- batched: many independent matrices in one persistent launch ---------

// Last matrix whose first global tile is <= t (matrices without tiles share
// their successor's first tile and are skipped this way).
__device__ __forceinline__ int64_t batch_matrix_of(const ascb_batch_item* __restrict__ items,
                                                   int64_t count, int64_t t) {
  int64_t lo = 0, hi = count - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(&items[mid].tile_base) <= t) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

__global__ void batch_bounds_kernel(const ascb_batch_item* __restrict__ items, int64_t count,
                                    int64_t* __restrict__ bounds, int64_t total_bounds) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total_bounds;
       e += step) {
    int64_t lo = 0, hi = count - 1;  // last matrix with bound_base <= e
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (__ldg(&items[mid].bound_base) <= e) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    const ascb_batch_item& it = items[lo];
    const int64_t next = lo + 1 < count ? __ldg(&items[lo + 1].bound_base) : total_bounds;
    const int64_t tiles = next - __ldg(&it.bound_base) - 1;
    const int64_t k = e - __ldg(&it.bound_base);
    bounds[e] = k >= tiles ? __ldg(&it.rows)
                           : first_row_at(it.ptr, __ldg(&it.rows), kRowWeight, k * kItems);
  }
}

template <typename T, bool EXACT, bool UNIT>
__global__ void __launch_bounds__(kThreads, EXACT ? kMinCtasExact : kMinCtasFast)
seg_batch_kernel(const ascb_batch_item* __restrict__ items, int64_t count,
                 const int64_t* __restrict__ bounds, int64_t total_tiles,
                 unsigned long long* __restrict__ queue, int chunk, T alpha, T beta) {
  __shared__ SegSmem<T> smem_all[kWarpsPerCta];
  const int lane = threadIdx.x & 31;
  SegSmem<T>& w = smem_all[threadIdx.x >> 5];
  int64_t tile_lo = 0, tile_hi = 0, bound_base = 0;
  const int64_t* ptr = nullptr;
  const int64_t* idx = nullptr;
  const T* val = nullptr;
  const T* x = nullptr;
  T* y = nullptr;
  int64_t incx = 1, incy = 1;
  for (;;) {
    unsigned long long t0 = 0;
    if (lane == 0) t0 = atomicAdd(queue, static_cast<unsigned long long>(chunk));
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= static_cast<unsigned long long>(total_tiles)) break;
    const int64_t t1 = static_cast<int64_t>(t0) + chunk < total_tiles
                           ? static_cast<int64_t>(t0) + chunk : total_tiles;
    for (int64_t t = static_cast<int64_t>(t0); t < t1; ++t) {
      if (t < tile_lo || t >= tile_hi) {
        const int64_t m = batch_matrix_of(items, count, t);
        const ascb_batch_item& it = items[m];
        tile_lo = __ldg(&it.tile_base);
        tile_hi = m + 1 < count ? __ldg(&items[m + 1].tile_base) : total_tiles;
        bound_base = __ldg(&it.bound_base);
        ptr = it.ptr;
        idx = it.idx;
        val = static_cast<const T*>(it.val);
        x = static_cast<const T*>(it.x);
        y = static_cast<T*>(it.y);
        incx = __ldg(&it.incx);
        incy = __ldg(&it.incy);
      }
      const int64_t k = bound_base + (t - tile_lo);
      const int64_t r0 = __ldg(bounds + k);
      const int nr = static_cast<int>(__ldg(bounds + k + 1) - r0);
      if (nr == 0) continue;
      const int64_t rb = lane < nr ? __ldg(ptr + r0 + lane) : 0;
      const int64_t re = lane < nr ? __ldg(ptr + r0 + lane + 1) : 0;
      seg_tile<T, EXACT, false, UNIT>(w, lane, ptr, idx, val, x, incx, y, incy, alpha, beta, r0, nr,
                                      rb, re);
    }
  }
}

// CTAs per SM at full occupancy, cached per device and per kernel (Tag
// distinguishes kernels with the same template arguments).
template <typename T, bool EXACT, bool STANDARD, bool UNIT, int Tag = 0, typename Kernel>
int resident(Kernel kernel) {
  static int cached[kMaxDevices] = {};
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return 1;
  if (cached[device] == 0) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, 0) != cudaSuccess ||
        n <= 0) {
      (void)cudaGetLastError();
      n = 1;
    }
    cached[device] = n;
  }
  return cached[device];
}

// 32-byte loads when both streamed arrays start on 32-byte boundaries.
inline bool aligned32(const ascb_csr* a) {
  return ((reinterpret_cast<uintptr_t>(a->idx) | reinterpret_cast<uintptr_t>(a->val)) & 31u) == 0;
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT, bool V32, int RPL>
int launch_v(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
             const ascb_vec* y, const int64_t* tile_row, int64_t ntiles, int sm_count) {
  auto kernel = seg_kernel<T, EXACT, STANDARD, UNIT, false, V32, RPL>;
  const int64_t warps_needed = (ntiles + 3) / 4;
  const int64_t ctas_needed = (warps_needed + kWarpsPerCta - 1) / kWarpsPerCta;
  const int64_t resident_ctas = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) *
                                resident<T, EXACT, STANDARD, UNIT, (V32 ? 4 : 0) + 16 * RPL>(kernel);
  const unsigned blocks = static_cast<unsigned>(
      ctas_needed < 1 ? 1 : (ctas_needed < resident_ctas ? ctas_needed : resident_ctas));
  kernel<<<blocks, kThreads, 0, stream>>>(
      a->ptr, a->idx, static_cast<const T*>(a->val), static_cast<const T*>(x->data), x->stride,
      static_cast<T*>(y->data), y->stride, alpha, beta, tile_row, ntiles, a->rows, a->nnz,
      SplitBlock{});
  return static_cast<int>(cudaGetLastError());
}

template <typename T, bool EXACT, bool STANDARD, bool UNIT, int RPL>
int launch(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
           const ascb_vec* y, const int64_t* tile_row, int64_t ntiles, int sm_count) {
  return aligned32(a)
             ? launch_v<T, EXACT, STANDARD, UNIT, true, RPL>(stream, a, alpha, beta, x, y,
                                                            tile_row, ntiles, sm_count)
             : launch_v<T, EXACT, STANDARD, UNIT, false, RPL>(stream, a, alpha, beta, x, y,
                                                             tile_row, ntiles, sm_count);
}

template <typename T, bool STANDARD, bool UNIT, bool V32, int RPL>
int launch_split_v(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
                   const ascb_vec* y, const int64_t* tile_row, int64_t ntiles, int sm_count,
                   const SplitBlock& split) {
  auto kernel = seg_kernel<T, false, STANDARD, UNIT, true, V32, RPL>;
  const int64_t warps_needed = (ntiles + 3) / 4;
  const int64_t ctas_needed = (warps_needed + kWarpsPerCta - 1) / kWarpsPerCta;
  const int per_sm = resident<T, false, STANDARD, UNIT, (V32 ? 5 : 2) + 16 * RPL>(kernel);
  const int64_t resident_ctas = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * per_sm;
  const unsigned blocks = static_cast<unsigned>(
      ctas_needed < 1 ? 1 : (ctas_needed < resident_ctas ? ctas_needed : resident_ctas));
  kernel<<<blocks, kThreads, 0, stream>>>(
      a->ptr, a->idx, static_cast<const T*>(a->val), static_cast<const T*>(x->data), x->stride,
      static_cast<T*>(y->data), y->stride, alpha, beta, tile_row, ntiles, a->rows, a->nnz, split);
  int rc = static_cast<int>(cudaGetLastError());
  if (rc != 0) return rc;
  auto tails = split_chunk_kernel<T, STANDARD, UNIT, V32>;
  const int tail_per_sm = resident<T, false, STANDARD, UNIT, V32 ? 6 : 3>(tails);
  tails<<<static_cast<unsigned>((sm_count > 0 ? sm_count : 148) * tail_per_sm), kThreads, 0,
          stream>>>(a->idx, static_cast<const T*>(a->val), static_cast<const T*>(x->data),
                    x->stride, static_cast<T*>(y->data), y->stride, alpha, beta, split);
  return static_cast<int>(cudaGetLastError());
}

template <typename T, bool STANDARD, bool UNIT, int RPL>
int launch_split(cudaStream_t stream, const ascb_csr* a, T alpha, T beta, const ascb_vec* x,
                 const ascb_vec* y, const int64_t* tile_row, int64_t ntiles, int sm_count,
                 const SplitBlock& split) {
  return aligned32(a)
             ? launch_split_v<T, STANDARD, UNIT, true, RPL>(stream, a, alpha, beta, x, y, tile_row,
                                                           ntiles, sm_count, split)
             : launch_split_v<T, STANDARD, UNIT, false, RPL>(stream, a, alpha, beta, x, y,
                                                            tile_row, ntiles, sm_count, split);
}

template <typename T, bool EXACT, int RPL>
int by_form(cudaStream_t s, int form, const ascb_csr* a, double alpha, double beta,
            const ascb_vec* x, const ascb_vec* y, const int64_t* tiles, int64_t n, int sm) {
  const bool unit = x->stride == 1 && y->stride == 1;
  const T al = static_cast<T>(alpha), be = static_cast<T>(beta);
  if (form == ASCB_STANDARD) {
    return unit ? launch<T, EXACT, true, true, RPL>(s, a, al, be, x, y, tiles, n, sm)
                : launch<T, EXACT, true, false, RPL>(s, a, al, be, x, y, tiles, n, sm);
  }
  return unit ? launch<T, EXACT, false, true, RPL>(s, a, al, be, x, y, tiles, n, sm)
              : launch<T, EXACT, false, false, RPL>(s, a, al, be, x, y, tiles, n, sm);
}

// Contracted tiles only (the merge partition's weight-1 tiles: RPL = 8).
template <int RPL>
int seg_rows_fast(void* stream, int dtype, int form, const ascb_csr* a, double alpha,
                  double beta, const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
                  int64_t ntiles, int sm_count) {
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return by_form<double, false, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                       sm_count);
  }
  return by_form<float, false, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles, sm_count);
}

template <int RPL>
int seg_rows(void* stream, int dtype, int form, int exact, const ascb_csr* a, double alpha,
             double beta, const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
             int64_t ntiles, int sm_count) {
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return exact ? by_form<double, true, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                              sm_count)
                 : by_form<double, false, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                               sm_count);
  }
  return exact ? by_form<float, true, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                           sm_count)
               : by_form<float, false, RPL>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                            sm_count);
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_spmv_seg(void* stream, int dtype, int form, int exact, const ascb_csr* a,
                             double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
                             const int64_t* tile_row, int64_t ntiles, int sm_count) {
  if (ntiles <= 0) return 0;
  return ascb::seg_rows<1>(stream, dtype, form, exact, a, alpha, beta, x, y, tile_row, ntiles,
                           sm_count);
}

extern "C" int64_t ascb_seg_tile_row_weight(void) { return ascb::kSegWeight; }
extern "C" int64_t ascb_seg_tile_items(void) {
  return ascb::tile_items<ascb::kMaxRowsPerLane>();
}
// The merge partition: one item per nonzero and one per row (weight 1), tiles
// of at most 250 items (up to 250 rows, 8 per lane).
extern "C" int64_t ascb_merge_tile_row_weight(void) { return 1; }
extern "C" int64_t ascb_merge_tile_items(void) { return ascb::tile_items<8>(); }

extern "C" int ascb_spmv_seg_w(void* stream, int dtype, int form, int exact, const ascb_csr* a,
                               double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
                               const int64_t* tile_row, int64_t ntiles, int64_t weight,
                               int sm_count) {
  if (ntiles <= 0) return 0;
  if (weight == ascb::kRowWeight) {
    return ascb::seg_rows<1>(stream, dtype, form, exact, a, alpha, beta, x, y, tile_row, ntiles,
                             sm_count);
  }
  if (weight == ascb::kSegWeight) {
    return ascb::seg_rows<ascb::kMaxRowsPerLane>(stream, dtype, form, exact, a, alpha, beta, x, y,
                                                 tile_row, ntiles, sm_count);
  }
  if (weight == 1 && !exact) {  // the merge partition (contracted only)
    return ascb::seg_rows_fast<8>(stream, dtype, form, a, alpha, beta, x, y, tile_row, ntiles,
                                  sm_count);
  }
  return static_cast<int>(cudaErrorInvalidValue);
}

extern "C" int ascb_spmv_seg_alignment(void) { return 16; }

namespace ascb {
namespace {

// Layout of a row-split block for `nnz` stored entries and tails longer than
// `split_min` (>= 256) positions: every split row has more than split_min
// tail positions, so at most nnz / (split_min + 1) + 1 entries, and at most
// nnz / 256 + entries chunks.
struct SplitLayout {
  int64_t entries, chunks;
  size_t done, table, head, partial, total;
};
SplitLayout split_layout(int64_t nnz, int64_t split_min) {
  auto up = [](size_t v) { return (v + 255) / 256 * 256; };
  SplitLayout l;
  l.entries = nnz / (split_min + 1) + 1;
  l.chunks = nnz / kItems + l.entries + 1;
  l.done = 256;
  l.table = up(l.done + static_cast<size_t>(l.entries) * sizeof(int));
  l.head = up(l.table + static_cast<size_t>(l.entries) * sizeof(SplitEntry));
  l.partial = up(l.head + static_cast<size_t>(l.entries) * 8);
  l.total = up(l.partial + static_cast<size_t>(l.chunks) * 8);
  return l;
}

template <typename T, int RPL>
int split_typed(cudaStream_t s, int form, const ascb_csr* a, double alpha, double beta,
                const ascb_vec* x, const ascb_vec* y, const int64_t* tiles, int64_t n, int sm,
                const SplitBlock& b) {
  const bool unit = x->stride == 1 && y->stride == 1;
  const T al = static_cast<T>(alpha), be = static_cast<T>(beta);
  if (form == ASCB_STANDARD) {
    return unit ? launch_split<T, true, true, RPL>(s, a, al, be, x, y, tiles, n, sm, b)
                : launch_split<T, true, false, RPL>(s, a, al, be, x, y, tiles, n, sm, b);
  }
  return unit ? launch_split<T, false, true, RPL>(s, a, al, be, x, y, tiles, n, sm, b)
              : launch_split<T, false, false, RPL>(s, a, al, be, x, y, tiles, n, sm, b);
}

}  // namespace
}  // namespace ascb

extern "C" size_t ascb_split_bytes(int64_t nnz, int64_t split_min) {
  if (split_min < ascb::kItems) split_min = ascb::kItems;
  return ascb::split_layout(nnz, split_min).total;
}

extern "C" int ascb_spmv_split(void* stream, int dtype, int form, const ascb_csr* a, double alpha,
                               double beta, const ascb_vec* x, const ascb_vec* y,
                               const int64_t* tile_row, int64_t ntiles, int64_t weight,
                               int64_t split_min, void* block, int sm_count) {
  if (ntiles <= 0) return 0;
  if (weight != ascb::kRowWeight && weight != ascb::kSegWeight) {
    return static_cast<int>(cudaErrorInvalidValue);
  }
  if (split_min < ascb::kItems) split_min = ascb::kItems;
  const ascb::SplitLayout l = ascb::split_layout(a->nnz, split_min);
  auto* base = static_cast<unsigned char*>(block);
  auto s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(block, 0, l.table, s);  // reservation word + finish counts
  if (e != cudaSuccess) return static_cast<int>(e);
  ascb::SplitBlock b;
  b.packed = reinterpret_cast<unsigned long long*>(base);
  b.done = reinterpret_cast<int*>(base + l.done);
  b.entries = reinterpret_cast<ascb::SplitEntry*>(base + l.table);
  b.head = base + l.head;
  b.partial = base + l.partial;
  b.max_entries = l.entries;
  b.max_chunks = l.chunks;
  b.split_min = split_min;
  constexpr int kR = ascb::kMaxRowsPerLane;
  if (weight == ascb::kSegWeight && kR > 1) {
    return dtype == ASCB_F64
               ? ascb::split_typed<double, kR>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                               sm_count, b)
               : ascb::split_typed<float, kR>(s, form, a, alpha, beta, x, y, tile_row, ntiles,
                                              sm_count, b);
  }
  return dtype == ASCB_F64 ? ascb::split_typed<double, 1>(s, form, a, alpha, beta, x, y, tile_row,
                                                          ntiles, sm_count, b)
                           : ascb::split_typed<float, 1>(s, form, a, alpha, beta, x, y, tile_row,
                                                         ntiles, sm_count, b);
}

namespace ascb {
namespace {

template <typename T, bool EXACT, bool UNIT>
int launch_batch(cudaStream_t s, const ascb_batch_item* items, int64_t count,
                 const int64_t* bounds, int64_t total_tiles, unsigned long long* queue, int chunk,
                 int ctas_per_sm, T alpha, T beta, int sm) {
  auto kernel = seg_batch_kernel<T, EXACT, UNIT>;
  int per_sm = ctas_per_sm;
  if (per_sm <= 0) per_sm = resident<T, EXACT, false, UNIT, 1>(kernel);
  const int64_t warps_needed = (total_tiles + chunk - 1) / chunk;
  const int64_t ctas_needed = (warps_needed + kWarpsPerCta - 1) / kWarpsPerCta;
  const int64_t cap = static_cast<int64_t>(sm > 0 ? sm : 148) * per_sm;
  const unsigned blocks =
      static_cast<unsigned>(ctas_needed < 1 ? 1 : (ctas_needed < cap ? ctas_needed : cap));
  kernel<<<blocks, kThreads, 0, s>>>(items, count, bounds, total_tiles, queue, chunk, alpha, beta);
  return static_cast<int>(cudaGetLastError());
}

template <typename T>
int batch_typed(cudaStream_t s, int exact, int unit, const ascb_batch_item* items, int64_t count,
                const int64_t* bounds, int64_t total_tiles, unsigned long long* queue, int chunk,
                int ctas, double alpha, double beta, int sm) {
  const T a = static_cast<T>(alpha), b = static_cast<T>(beta);
  if (exact) {
    return unit ? launch_batch<T, true, true>(s, items, count, bounds, total_tiles, queue, chunk,
                                              ctas, a, b, sm)
                : launch_batch<T, true, false>(s, items, count, bounds, total_tiles, queue, chunk,
                                               ctas, a, b, sm);
  }
  return unit ? launch_batch<T, false, true>(s, items, count, bounds, total_tiles, queue, chunk,
                                             ctas, a, b, sm)
              : launch_batch<T, false, false>(s, items, count, bounds, total_tiles, queue, chunk,
                                              ctas, a, b, sm);
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_batch_tile_bounds(void* stream, const ascb_batch_item* items, int64_t count,
                                      int64_t* bounds, int64_t total_bounds, int sm_count) {
  if (count <= 0 || total_bounds <= 0) return 0;
  int64_t blocks = (total_bounds + 255) / 256;
  const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
  if (blocks > cap) blocks = cap;
  ascb::batch_bounds_kernel<<<static_cast<unsigned>(blocks), 256, 0,
                              static_cast<cudaStream_t>(stream)>>>(items, count, bounds,
                                                                  total_bounds);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_spmv_seg_batch(void* stream, int dtype, int exact, int unit,
                                   const ascb_batch_item* items, int64_t count,
                                   const int64_t* bounds, int64_t total_tiles,
                                   unsigned long long* queue, int chunk, int ctas_per_sm,
                                   double alpha, double beta, int sm_count) {
  if (count <= 0 || total_tiles <= 0) return 0;
  if (chunk < 1) chunk = 1;
  auto s = static_cast<cudaStream_t>(stream);
  if (dtype == ASCB_F64) {
    return ascb::batch_typed<double>(s, exact, unit, items, count, bounds, total_tiles, queue,
                                     chunk, ctas_per_sm, alpha, beta, sm_count);
  }
  return ascb::batch_typed<float>(s, exact, unit, items, count, bounds, total_tiles, queue, chunk,
                                  ctas_per_sm, alpha, beta, sm_count);
}
