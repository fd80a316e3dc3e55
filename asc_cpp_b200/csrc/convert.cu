// Device format conversions for sm_100a: CSR <-> CSC and coordinates ->
// CSR / CSC, and the transposed structure that deterministic transposed
// products run on.
//
// Each of them is one STABLE sort of entry positions by the entry's new outer
// index.  That is the order in which the reference's host conversions emit
// entries (CompressedSparseArray::FromCoordinate, compressed.h:1082-1131, and
// FromCompressed, :1151-1221, scan the source in stored order once per
// destination outer index), and the order in which the reference's standard
// transposed products accumulate (blas.h:1241-1256, outer then inner).
//
// The sort is a least-significant-digit radix sort with 8-bit digits over
// tiles of 4096 entries:
//   * count:   each tile histograms its digits in shared memory (the counts
//              do not depend on the order of the atomics);
//   * scan:    an exclusive scan of the digit-major (digit, tile) count table
//              gives every digit of every tile its first output slot;
//   * scatter: each warp ranks its 512 entries 32 at a time, in stored order,
//              with __match_any_sync; the tile's warps are offset by a scan of
//              their per-digit counts, so equal digits keep their input order.
// ceil(bits(limit - 1) / 8) passes; each reads and writes a key and a payload
// (16 bytes per entry).  The bucket offsets are a histogram of the whole key
// followed by the same scan.  Everything is integer work, so the results are
// exact by construction and independent of scheduling.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortPer = 16;                                 // entries per thread
constexpr int64_t kSortTile = int64_t{kSortThreads} * kSortPer;  // 4096
constexpr int kWarpSpan = 32 * kSortPer;                     // 512 per warp
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 8;
constexpr int64_t kScanChunk = int64_t{kScanThreads} * kScanPer;  // 8192

std::size_t Round256(std::size_t v) { return (v + 255) / 256 * 256; }

__device__ __forceinline__ int digit_of(int64_t key, int shift) {
  return static_cast<int>((static_cast<uint64_t>(key) >> shift) & (kRadix - 1));
}

// ---- exclusive scan of int64 arrays (three launches, any length) ----------

// Exclusive scan of one value per thread over the block; *total receives the
// block's sum.  `sums` holds 32 entries of shared memory.
__device__ int64_t block_exclusive(int64_t v, int64_t* sums, int64_t* total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  int64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int nwarps = static_cast<int>(blockDim.x >> 5);
    int64_t w = lane < nwarps ? sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    sums[lane] = w;
  }
  __syncthreads();
  const int64_t prefix = warp > 0 ? sums[warp - 1] : 0;
  *total = sums[31];
  __syncthreads();  // sums is reused by the caller's next round
  return prefix + inc - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce(const int64_t* __restrict__ in,
                                                            int64_t n,
                                                            int64_t* __restrict__ partial) {
  __shared__ int64_t sums[32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanChunk + threadIdx.x * kScanPer;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) s += in[base + k];
  }
  int64_t total = 0;
  (void)block_exclusive(s, sums, &total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// One block: exclusive scan of the m chunk sums in place.
__global__ void __launch_bounds__(kScanThreads) scan_partials(int64_t* __restrict__ partial,
                                                              int64_t m) {
  __shared__ int64_t sums[32];
  int64_t carry = 0;
  for (int64_t base = 0; base < m; base += kScanThreads) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < m ? partial[i] : 0;
    int64_t total = 0;
    const int64_t ex = block_exclusive(v, sums, &total);
    if (i < m) partial[i] = carry + ex;
    carry += total;
  }
}

// out may alias in: every thread reads its 8 values before any write, and
// chunks of different threads are disjoint.
__global__ void __launch_bounds__(kScanThreads) scan_apply(const int64_t* in, int64_t n,
                                                           const int64_t* __restrict__ partial,
                                                           int64_t* out) {
  __shared__ int64_t sums[32];
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanChunk + threadIdx.x * kScanPer;
  int64_t v[kScanPer];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  int64_t total = 0;
  int64_t run = block_exclusive(s, sums, &total) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

std::size_t ScanPartialBytes(int64_t n) {
  return Round256(static_cast<std::size_t>((n + kScanChunk - 1) / kScanChunk + 1) * 8);
}

cudaError_t ExclusiveScan(cudaStream_t stream, int64_t* data, int64_t n, int64_t* partial) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + kScanChunk - 1) / kScanChunk;
  scan_reduce<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(data, n, partial);
  scan_partials<<<1, kScanThreads, 0, stream>>>(partial, blocks);
  scan_apply<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(data, n, partial, data);
  return cudaGetLastError();
}

// ---- radix passes ---------------------------------------------------------

__global__ void __launch_bounds__(kSortThreads)
radix_count(const int64_t* __restrict__ keys, int64_t kstride, int64_t n, int shift,
            int64_t* __restrict__ table, int64_t tiles) {
  __shared__ int counts[kRadix];
  for (int i = threadIdx.x; i < kRadix; i += kSortThreads) counts[i] = 0;
  __syncthreads();
  const int64_t begin = static_cast<int64_t>(blockIdx.x) * kSortTile;
#pragma unroll 4
  for (int j = 0; j < kSortPer; ++j) {
    const int64_t e = begin + j * kSortThreads + threadIdx.x;
    if (e < n) atomicAdd(&counts[digit_of(__ldg(keys + e * kstride), shift)], 1);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
    table[d * tiles + blockIdx.x] = counts[d];
  }
}

// pay == nullptr: the payload is the entry's position.  keys_out == nullptr:
// keys are not written (last pass).
__global__ void __launch_bounds__(kSortThreads)
radix_scatter(const int64_t* __restrict__ keys, int64_t kstride, const int64_t* __restrict__ pay,
              int64_t n, int shift, const int64_t* __restrict__ table, int64_t tiles,
              int64_t* __restrict__ keys_out, int64_t* __restrict__ pay_out) {
  __shared__ int warp_count[kSortWarps][kRadix];
  __shared__ int64_t tile_start[kRadix];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) {
    (&warp_count[0][0])[i] = 0;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  const int64_t begin = static_cast<int64_t>(blockIdx.x) * kSortTile + warp * kWarpSpan;
  int64_t key[kSortPer];
  int64_t val[kSortPer];
  int rank[kSortPer];
#pragma unroll
  for (int j = 0; j < kSortPer; ++j) {
    const int64_t e = begin + j * 32 + lane;
    const bool ok = e < n;
    key[j] = ok ? __ldg(keys + e * kstride) : 0;
    val[j] = ok ? (pay != nullptr ? __ldg(pay + e) : e) : 0;
    const int d = ok ? digit_of(key[j], shift) : kRadix;  // kRadix: no entry
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int before = ok ? warp_count[warp][d] : 0;
    rank[j] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && (peers & lt) == 0u) warp_count[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
    int s = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const int c = warp_count[w][d];
      warp_count[w][d] = s;
      s += c;
    }
    tile_start[d] = table[d * tiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortPer; ++j) {
    const int64_t e = begin + j * 32 + lane;
    if (e < n) {
      const int d = digit_of(key[j], shift);
      const int64_t q = tile_start[d] + warp_count[warp][d] + rank[j];
      if (keys_out != nullptr) keys_out[q] = key[j];
      pay_out[q] = val[j];
    }
  }
}

// counts[k] += 1 for every key k in [0, limit); other keys are ignored.
__global__ void key_count(const int64_t* __restrict__ keys, int64_t kstride, int64_t n,
                          int64_t limit, int64_t* __restrict__ counts) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += step) {
    const int64_t k = __ldg(keys + e * kstride);
    if (k >= 0 && k < limit) {
      atomicAdd(reinterpret_cast<unsigned long long*>(counts + k), 1ull);
    }
  }
}

// out[q] = r for every entry q of outer index r (one warp per outer index).
__global__ void outer_of_entries(const int64_t* __restrict__ ptr, int64_t outer,
                                 int64_t* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < outer;
       r += warps) {
    const int64_t b = __ldg(ptr + r);
    const int64_t e = __ldg(ptr + r + 1);
    for (int64_t q = b + lane; q < e; q += 32) out[q] = r;
  }
}

struct alignas(16) Bytes16 {
  uint64_t lo, hi;
};

template <typename V>
__global__ void permute_entries(const int64_t* __restrict__ perm, int64_t n,
                                const int64_t* __restrict__ other, int64_t ostride,
                                int64_t* __restrict__ idx_out, const V* __restrict__ val_in,
                                V* __restrict__ val_out) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n;
       j += step) {
    const int64_t p = __ldg(perm + j);
    if (idx_out != nullptr) idx_out[j] = __ldg(other + p * ostride);
    if (val_out != nullptr) val_out[j] = val_in[p];
  }
}

unsigned GridFor(int64_t n, int threads, int sm_count) {
  const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
  int64_t blocks = (n + threads - 1) / threads;
  if (blocks > cap) blocks = cap;
  return static_cast<unsigned>(blocks < 1 ? 1 : blocks);
}

int Passes(int64_t limit) {
  int bits = 0;
  for (uint64_t v = limit > 1 ? static_cast<uint64_t>(limit - 1) : 0; v != 0; v >>= 1) ++bits;
  const int p = (bits + kRadixBits - 1) / kRadixBits;
  return p < 1 ? 1 : p;
}

struct SortLayout {
  std::size_t keys[2], pay[2], table, partial, total;
};

SortLayout Layout(int64_t n, int64_t limit) {
  SortLayout l{};
  const int64_t tiles = (n + kSortTile - 1) / kSortTile;
  const std::size_t entries = Round256(static_cast<std::size_t>(n > 0 ? n : 1) * 8);
  std::size_t at = 0;
  for (int i = 0; i < 2; ++i) {
    l.keys[i] = at;
    at += entries;
  }
  for (int i = 0; i < 2; ++i) {
    l.pay[i] = at;
    at += entries;
  }
  l.table = at;
  const int64_t table_n = int64_t{kRadix} * (tiles > 0 ? tiles : 1);
  at += Round256(static_cast<std::size_t>(table_n) * 8);
  l.partial = at;
  at += ScanPartialBytes(table_n > limit + 1 ? table_n : limit + 1);
  l.total = at;
  return l;
}

}  // namespace
}  // namespace ascb

extern "C" size_t ascb_sort_workspace_bytes(int64_t n, int64_t limit) {
  return ascb::Layout(n, limit).total;
}

extern "C" int ascb_stable_sort(void* stream_ptr, const int64_t* keys, int64_t kstride, int64_t n,
                                int64_t limit, int64_t* offsets, int64_t* perm, void* workspace) {
  using namespace ascb;
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  auto* ws = static_cast<unsigned char*>(workspace);
  const SortLayout l = Layout(n, limit);
  int64_t* partial = reinterpret_cast<int64_t*>(ws + l.partial);
  // bucket offsets: histogram of the whole key, then an exclusive scan
  cudaError_t e = cudaMemsetAsync(offsets, 0, static_cast<std::size_t>(limit + 1) * 8, stream);
  if (e != cudaSuccess) return static_cast<int>(e);
  if (n > 0) {
    key_count<<<GridFor(n, 256, 148), 256, 0, stream>>>(keys, kstride, n, limit, offsets);
  }
  e = ExclusiveScan(stream, offsets, limit + 1, partial);
  if (e != cudaSuccess || n == 0) return static_cast<int>(e);

  const int64_t tiles = (n + kSortTile - 1) / kSortTile;
  int64_t* table = reinterpret_cast<int64_t*>(ws + l.table);
  int64_t* kbuf[2] = {reinterpret_cast<int64_t*>(ws + l.keys[0]),
                      reinterpret_cast<int64_t*>(ws + l.keys[1])};
  int64_t* pbuf[2] = {reinterpret_cast<int64_t*>(ws + l.pay[0]),
                      reinterpret_cast<int64_t*>(ws + l.pay[1])};
  const int passes = Passes(limit);
  for (int p = 0; p < passes; ++p) {
    const int64_t* kin = p == 0 ? keys : kbuf[(p - 1) & 1];
    const int64_t ks = p == 0 ? kstride : 1;
    const int64_t* pin = p == 0 ? nullptr : pbuf[(p - 1) & 1];
    const bool last = p + 1 == passes;
    const int shift = p * kRadixBits;
    radix_count<<<static_cast<unsigned>(tiles), kSortThreads, 0, stream>>>(kin, ks, n, shift,
                                                                          table, tiles);
    e = ExclusiveScan(stream, table, int64_t{kRadix} * tiles, partial);
    if (e != cudaSuccess) return static_cast<int>(e);
    radix_scatter<<<static_cast<unsigned>(tiles), kSortThreads, 0, stream>>>(
        kin, ks, pin, n, shift, table, tiles, last ? nullptr : kbuf[p & 1],
        last ? perm : pbuf[p & 1]);
  }
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_outer_of_entries(void* stream, const int64_t* ptr, int64_t outer, int64_t* out,
                                     int sm_count) {
  if (outer <= 0) return 0;
  const unsigned blocks = ascb::GridFor(outer * 32, 256, sm_count);
  ascb::outer_of_entries<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(ptr, outer, out);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int ascb_permute_entries(void* stream_ptr, const int64_t* perm, int64_t n,
                                    const int64_t* other, int64_t ostride, int64_t* idx_out,
                                    const void* val_in, void* val_out, int elem_bytes,
                                    int sm_count) {
  using namespace ascb;
  if (n <= 0) return 0;
  auto stream = static_cast<cudaStream_t>(stream_ptr);
  const unsigned blocks = GridFor(n, 256, sm_count);
  switch (elem_bytes) {
    case 4:
      permute_entries<uint32_t><<<blocks, 256, 0, stream>>>(
          perm, n, other, ostride, idx_out, static_cast<const uint32_t*>(val_in),
          static_cast<uint32_t*>(val_out));
      break;
    case 8:
      permute_entries<uint64_t><<<blocks, 256, 0, stream>>>(
          perm, n, other, ostride, idx_out, static_cast<const uint64_t*>(val_in),
          static_cast<uint64_t*>(val_out));
      break;
    case 16:
      permute_entries<Bytes16><<<blocks, 256, 0, stream>>>(
          perm, n, other, ostride, idx_out, static_cast<const Bytes16*>(val_in),
          static_cast<Bytes16*>(val_out));
      break;
    default:
      return static_cast<int>(cudaErrorInvalidValue);
  }
  return static_cast<int>(cudaGetLastError());
}
