// Block-sparse SpMM on the tensor cores (tcgen05, kind::tf32) for sm_100a.
//
// For CSR matrices made of dense 16 x 16 blocks -- every block row's sixteen
// rows store the same column list, made of whole, aligned groups of sixteen
// columns (ascb_block16_check) -- with FP32 values and row-major B and C:
//     C += alpha * A * B.
// A CTA takes a block row and a chunk of up to 128 right-hand sides at a
// time and accumulates, in tensor memory,
//     D (128 x 16) = sum over the block row's blocks of  B_blk^T (128 x 16) . A_blk^T
// i.e. D[m][n] = sum_kk B[16 bc + kk][m] A_blk[n][kk] = (A B)[16 br + n][m].
// The product of a block is one MMA of M = 128 (right-hand sides, zero-padded),
// N = 16 (rows of the block), K = 16 (two K = 8 steps).  Both operands are
// staged in shared memory in the canonical K-major, 64-byte-swizzle layout
// (rows of 16 values = 64 bytes; the 16-byte chunk c of row r sits at chunk
// c ^ ((r >> 1) & 3)), written by the threads from registers: the A block's
// rows are read straight from the CSR value array (each row's 16 values are
// contiguous there), B's rows are read coalesced and transposed on the way.
//
// Precision: FP32 inputs are split as a = hi + lo with hi = a truncated to
// TF32 and lo = a - hi (exact), and each block contributes
//     hi_B hi_A + hi_B lo_A + lo_B hi_A
// (three MMAs into the same accumulator), so the result keeps close to FP32
// accuracy: |c - c_exact| <= (n + 64) 2^-22 |alpha| sum_k |a_k b_k| + 2^-23 |c0|
// per output, n = stored entries in the row (tests check this bound).
//
// B tiles: a pre-pass (bt_tiles_kernel, once per product) writes, for every
// block column and 128-column chunk of B, the two 8 KB shared-memory images
// hi and lo of B_blk^T, so a stage's B operand arrives as two TMA bulk copies
// (cp.async.bulk) of the chunk's `width` rows (16 KB at 128 right-hand sides,
// 1 KB at 8) from L2 -- no transposes, splits or LSU traffic for B in the
// main kernel.
//
// Pipeline: four producer warps each own one shared-memory stage and fill it
// for the blocks whose running index is their warp number mod 4: lane 0
// issues the B tile's bulk copy (expect-tx on the stage's `full` barrier),
// the lanes split the block's A rows (loaded before the stage wait) into
// hi / lo and arrive; one thread issues the MMAs as stages fill (mbarriers
// full / empty); two 16-column accumulators alternate between block rows so
// the epilogue of one overlaps the MMAs of the next.
// Every wait is bounded: one that runs out records 1 in *status, tells the
// other roles to stop (a shared flag), and the CTA waits (bounded) for its own
// MMAs before it frees its tensor memory.
#include <cstddef>

#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kProducerWarps = 4;
constexpr int kProducerThreads = kProducerWarps * 32;
constexpr int kThreads = kProducerThreads + 32;  // + the MMA warp
constexpr int kStages = kProducerWarps;          // one stage per producer warp
constexpr int kM = 128;        // right-hand sides per pass
constexpr int kB = 16;         // block size
constexpr int kTmemCols = 32;  // two accumulators of 16 columns
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kSuspendNs = 1000;

struct alignas(1024) Stage {
  float bt_hi[kM * kB];  // B^T tile, 128 rows x 16, K-major SW64 (8 KB)
  float bt_lo[kM * kB];
  float a_hi[kB * kB];   // A block, 16 rows x 16 (1 KB)
  float a_lo[kB * kB];
};

static_assert(offsetof(Stage, bt_lo) == offsetof(Stage, bt_hi) + sizeof(float) * kM * kB,
              "a stage's B^T images are adjacent: one bulk copy fills both");

struct Smem {
  Stage stage[kStages];
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t dfull[2];
  uint64_t dempty[2];
  uint64_t done;
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of 16-byte chunk c of row r in a K-major 64-byte-swizzle tile
__device__ __forceinline__ uint32_t swz(uint32_t r, uint32_t c) {
  return r * 64u + ((c ^ ((r >> 1) & 3u)) << 4);
}

// shared memory descriptor: K-major, SWIZZLE_64B, 8-row groups 512 B apart
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3fffu);  // start address
  d |= static_cast<uint64_t>(1u) << 16;                // leading offset (unused here)
  d |= static_cast<uint64_t>(512u >> 4) << 32;         // stride offset
  d |= static_cast<uint64_t>(1u) << 46;                // descriptor version
  d |= static_cast<uint64_t>(4u) << 61;                // SWIZZLE_64B
  return d;
}

// instruction descriptor: D F32, A/B TF32, both K-major, N = 16, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void split(float4 v, float4& hi, float4& lo) {
  const uint32_t m = 0xffffe000u;
  hi.x = __uint_as_float(__float_as_uint(v.x) & m);
  hi.y = __uint_as_float(__float_as_uint(v.y) & m);
  hi.z = __uint_as_float(__float_as_uint(v.z) & m);
  hi.w = __uint_as_float(__float_as_uint(v.w) & m);
  lo.x = v.x - hi.x;
  lo.y = v.y - hi.y;
  lo.z = v.z - hi.z;
  lo.w = v.w - hi.w;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::
                   "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n .reg .b64 st;\n"
      " mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Pre-pass: tile (bc, ch) of B^T for block column bc and right-hand sides
// [128 ch, 128 ch + 128): element (m, kk) = B(16 bc + kk, 128 ch + m) (0 past
// k), as the K-major 64-byte-swizzle image of a stage (hi, then lo).  One
// thread per (tile, m, 16-byte chunk).
constexpr int kTileFloats = kM * kB;  // 2048 per image
__global__ void __launch_bounds__(256)
bt_tiles_kernel(const float* __restrict__ b, int64_t ldb, int64_t k, int64_t b_rows,
                int64_t col_blocks, int64_t chunks, float* __restrict__ tiles) {
  const int64_t total = col_blocks * chunks * kM * 4;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += step) {
    const int m = static_cast<int>(i % kM);
    const int cq = static_cast<int>((i / kM) % 4);
    const int64_t tile = i / (kM * 4);  // bc * chunks + ch
    const int64_t bc = tile / chunks;
    const int64_t col = (tile - bc * chunks) * kM + m;
    if (col >= k) continue;  // rows past k are never copied (see the producers)
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int64_t row = bc * kB + cq * 4 + e;
      v[e] = row < b_rows ? __ldg(b + row * ldb + col) : 0.0f;
    }
    float4 hi, lo;
    split(make_float4(v[0], v[1], v[2], v[3]), hi, lo);
    unsigned char* base = reinterpret_cast<unsigned char*>(tiles + tile * 2 * kTileFloats);
    *reinterpret_cast<float4*>(base + swz(m, cq)) = hi;
    *reinterpret_cast<float4*>(base + kTileFloats * 4 + swz(m, cq)) = lo;
  }
}

// bounded wait for phase `parity` of `bar`; false if it ran out or another
// role of the CTA gave up (*abort)
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity, const int* abort) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (ok) return true;
    if (abort != nullptr && *reinterpret_cast<const volatile int*>(abort)) return false;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&d)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
        "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]),
        "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Roles: warps 0..3 produce (warp p stages the blocks whose running index is
// p mod 4, in stage p, and runs the epilogue for TMEM lanes 32p..32p+31);
// warp 4 follows the same sequence and its lane 0 issues the MMAs.
// Barriers: full[p] (32 producer lanes arrive) -> MMAs -> empty[p]
// (tcgen05.commit); at the end of a block row the
// MMA thread commits dfull[a] for accumulator a, the producers read D and
// arrive on dempty[a] (128 arrivals).
__global__ void __launch_bounds__(kThreads)
block16_tc_kernel(const int64_t* __restrict__ ptr, const int64_t* __restrict__ idx,
                  const float* __restrict__ val, int64_t block_rows,
                  const float* __restrict__ tiles, float* __restrict__ c, int64_t ldc, int64_t k,
                  float alpha, int* status) {
  extern __shared__ unsigned char smem_raw[];
  Smem& s = *reinterpret_cast<Smem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const int t = threadIdx.x;
  const int warp = t >> 5;
  const int lane = t & 31;
  if (t == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&s.full[i], 32);
      mbar_init(&s.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.dfull[i], 1);
      mbar_init(&s.dempty[i], kProducerThreads);
    }
    mbar_init(&s.done, 1);
    s.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&s.tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s.tmem;
  const int64_t chunks = (k + kM - 1) / kM;
  const int64_t items = block_rows * chunks;
  bool failed = false;

  if (warp < kProducerWarps) {
    // ---------------- producers ----------------
    const int p = warp;
    unsigned char* stage = reinterpret_cast<unsigned char*>(&s.stage[p]);
    unsigned char* bt_hi = stage + offsetof(Stage, bt_hi);  // bt_lo follows it
    unsigned char* a_hi = stage + offsetof(Stage, a_hi);
    unsigned char* a_lo = stage + offsetof(Stage, a_lo);
    // this lane's A chunks: rows lane/4 and lane/4 + 8, 16-byte chunk lane%4
    const int ar = lane >> 2;
    const int ac = lane & 3;
    uint32_t it = 0, itm = 0, uses = 0;
    for (int64_t item = blockIdx.x; item < items && !failed; item += gridDim.x) {
      const int64_t br = item / chunks;
      const int64_t ch = item - br * chunks;
      const int64_t m0 = ch * kM;
      const int64_t width = k - m0 < kM ? k - m0 : kM;
      const int64_t p0 = __ldg(ptr + br * kB);
      const int64_t nblk = (__ldg(ptr + br * kB + 1) - p0) / kB;
      if (nblk == 0) continue;  // empty block row: C unchanged
      const float* a0 = val + __ldg(ptr + br * kB + ar) + ac * 4;
      const float* a1 = val + __ldg(ptr + br * kB + ar + 8) + ac * 4;
      for (int64_t j = 0; j < nblk; ++j, ++it) {
        if ((it & 3u) != static_cast<uint32_t>(p)) continue;
        // the block's A loads go out before the wait for the stage, so their
        // latency overlaps the MMAs still reading it
        const int64_t bc = __ldg(idx + p0 + j * kB) >> 4;
        const float4 va0 = __ldg(reinterpret_cast<const float4*>(a0 + j * kB));
        const float4 va1 = __ldg(reinterpret_cast<const float4*>(a1 + j * kB));
        if (uses > 0 && !wait_bar(&s.empty[p], (uses - 1) & 1u, &s.abort)) {
          failed = true;
          break;
        }
        if (lane == 0) {
          // rows [0, width) of B^T hi and lo of (bc, ch): a row is 64 bytes and
          // the swizzle permutes chunks only within a row, so the images'
          // first `width` rows are contiguous.  Rows past width keep stale data:
          // they feed only rows of D past width, which the epilogue never stores.
          const uint32_t bytes = static_cast<uint32_t>(width) * kB * 4;
          const float* src = tiles + (bc * chunks + ch) * 2 * kTileFloats;
          mbar_expect_tx(&s.full[p], 2 * bytes);
          bulk_copy(bt_hi, src, bytes, &s.full[p]);
          bulk_copy(bt_hi + kTileFloats * 4, src + kTileFloats, bytes, &s.full[p]);
        }
        float4 hi, lo;
        split(va0, hi, lo);
        *reinterpret_cast<float4*>(a_hi + swz(ar, ac)) = hi;
        *reinterpret_cast<float4*>(a_lo + swz(ar, ac)) = lo;
        split(va1, hi, lo);
        *reinterpret_cast<float4*>(a_hi + swz(ar + 8, ac)) = hi;
        *reinterpret_cast<float4*>(a_lo + swz(ar + 8, ac)) = lo;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(&s.full[p]);
        ++uses;
      }
      if (failed) break;
      // epilogue: this warp's quarter of D once the block row's MMAs are done
      const uint32_t a = itm & 1u;
      if (!wait_bar(&s.dfull[a], (itm >> 1) & 1u, &s.abort)) {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      uint32_t d[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(p * 32) << 16) + a * kB, d);
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      mbar_arrive(&s.dempty[a]);
      const int64_t m = p * 32 + lane;
      if (m < width) {
#pragma unroll
        for (int n = 0; n < kB; ++n) {
          float* cp = c + (br * kB + n) * ldc + m0 + m;
          *cp = fmaf(alpha, __uint_as_float(d[n]), *cp);
        }
      }
      ++itm;
    }
  } else {
    // ---------------- MMA issuer (warp 4: every lane waits, lane 0 issues) ----
    uint32_t it = 0, itm = 0;
    for (int64_t item = blockIdx.x; item < items && !failed; item += gridDim.x) {
      const int64_t br = item / chunks;
      const int64_t p0 = __ldg(ptr + br * kB);
      const int64_t nblk = (__ldg(ptr + br * kB + 1) - p0) / kB;
      if (nblk == 0) continue;
      const uint32_t a = itm & 1u;
      if (itm >= 2 && !wait_bar(&s.dempty[a], ((itm >> 1) - 1) & 1u, &s.abort)) {
        failed = true;
        break;
      }
      for (int64_t j = 0; j < nblk; ++j, ++it) {
        const uint32_t st = it & 3u;
        if (!wait_bar(&s.full[st], (it >> 2) & 1u, &s.abort)) {
          failed = true;
          break;
        }
        if (lane == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t base = smem_u32(&s.stage[st]);
          const uint32_t bh = base + offsetof(Stage, bt_hi);
          const uint32_t bl = base + offsetof(Stage, bt_lo);
          const uint32_t ah = base + offsetof(Stage, a_hi);
          const uint32_t al = base + offsetof(Stage, a_lo);
          const uint32_t pa[3] = {bh, bh, bl};
          const uint32_t pb[3] = {ah, al, ah};
#pragma unroll
          for (int q = 0; q < 3; ++q) {
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              const uint32_t acc = (j > 0 || q > 0 || ks > 0) ? 1u : 0u;
              mma_tf32(tmem + a * kB, sdesc(pa[q] + ks * 32), sdesc(pb[q] + ks * 32), acc);
            }
          }
          commit(&s.empty[st]);
        }
        __syncwarp();
      }
      if (failed) break;
      if (lane == 0) commit(&s.dfull[a]);
      __syncwarp();
      ++itm;
    }
    // every MMA of this CTA has completed once `done` fires
    if (lane == 0) commit(&s.done);
    __syncwarp();
    if (!wait_bar(&s.done, 0u, nullptr)) failed = true;
  }
  if (failed) {
    *reinterpret_cast<volatile int*>(&s.abort) = 1;
    if (status != nullptr) atomicExch(status, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// Block structure check (rows a multiple of 16, checked by the host): one warp
// per block row; sets *bad on any block row that breaks the 16 x 16
// dense-block pattern.
__global__ void block16_check_kernel(const int64_t* __restrict__ ptr,
                                     const int64_t* __restrict__ idx, int64_t block_rows,
                                     int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t br = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
       br < block_rows; br += warps) {
    const int64_t p0 = __ldg(ptr + br * kB);
    const int64_t len = __ldg(ptr + br * kB + 1) - p0;
    bool good = len % kB == 0;
    for (int i = 1; i < kB && good; ++i) {
      good = __ldg(ptr + br * kB + i + 1) - __ldg(ptr + br * kB + i) == len;
    }
    for (int64_t q = lane; q < len && good; q += 32) {
      const int64_t col = __ldg(idx + p0 + q);
      const int64_t head = __ldg(idx + p0 + (q & ~int64_t{kB - 1}));
      good = (head & (kB - 1)) == 0 && col == head + (q & (kB - 1));
      for (int i = 1; i < kB && good; ++i) {
        good = __ldg(idx + __ldg(ptr + br * kB + i) + q) == col;
      }
    }
    if (!__all_sync(0xffffffffu, good) && lane == 0) atomicExch(bad, 1);
  }
}

}  // namespace
}  // namespace ascb

extern "C" int ascb_block16_check(void* stream, const ascb_csr* a, int* bad, int sm_count) {
  auto s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int), s);
  if (e != cudaSuccess) return static_cast<int>(e);
  const int64_t block_rows = a->rows / 16;
  if (block_rows > 0) {
    int64_t blocks = (block_rows * 32 + 255) / 256;
    const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
    if (blocks > cap) blocks = cap;
    ascb::block16_check_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(a->ptr, a->idx,
                                                                            block_rows, bad);
  }
  return static_cast<int>(cudaGetLastError());
}

extern "C" size_t ascb_block16_tc_smem(void) { return sizeof(ascb::Smem) + 1024; }

extern "C" size_t ascb_block16_tiles_bytes(int64_t cols, int64_t k) {
  const int64_t chunks = (k + ascb::kM - 1) / ascb::kM;
  return static_cast<size_t>((cols + ascb::kB - 1) / ascb::kB) * static_cast<size_t>(chunks) * 2 *
         ascb::kTileFloats * sizeof(float);
}

extern "C" int ascb_spmm_block16_tc(void* stream, const ascb_csr* a, int64_t k, const float* b,
                                    int64_t ldb, float* c, int64_t ldc, float alpha,
                                    float* tiles, int* status, int sm_count) {
  using namespace ascb;
  if (a->rows <= 0 || k <= 0) return 0;
  const int64_t col_blocks = (a->cols + kB - 1) / kB;  // B rows past cols read as 0
  const int64_t chunks = (k + kM - 1) / kM;
  if (col_blocks > 0) {
    const int64_t work = col_blocks * chunks * kM * 4;
    int64_t blocks = (work + 255) / 256;
    const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * 8;
    if (blocks > cap) blocks = cap;
    bt_tiles_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        b, ldb, k, a->cols, col_blocks, chunks, tiles);
    const cudaError_t pe = cudaGetLastError();
    if (pe != cudaSuccess) return static_cast<int>(pe);
  }
  const size_t smem = ascb_block16_tc_smem();
  cudaError_t e = cudaFuncSetAttribute(
      block16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e == cudaSuccess) {
    // all of the unified L1/shared storage as shared memory: three CTAs fit
    e = cudaFuncSetAttribute(block16_tc_kernel,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  }
  if (e != cudaSuccess) return static_cast<int>(e);
  const int64_t block_rows = a->rows / 16;
  const int64_t items = block_rows * chunks;
  // CTAs per SM: the shared-memory limit (three at 75 KB each); the register
  // file (126 x 160 per CTA) allows more
  int device = 0, sm_smem = 0, reserved = 0;
  int per_sm = 1;
  if (cudaGetDevice(&device) == cudaSuccess &&
      cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) ==
          cudaSuccess &&
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) ==
          cudaSuccess) {
    const int fit = sm_smem / static_cast<int>(smem + static_cast<size_t>(reserved));
    per_sm = fit > 1 ? fit : 1;
  } else {
    (void)cudaGetLastError();
  }
  const int64_t cap = static_cast<int64_t>(sm_count > 0 ? sm_count : 148) * per_sm;
  const unsigned grid = static_cast<unsigned>(items < cap ? (items > 0 ? items : 1) : cap);
  block16_tc_kernel<<<grid, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(
      a->ptr, a->idx, static_cast<const float*>(a->val), block_rows, tiles, c, ldc, k, alpha,
      status);
  return static_cast<int>(cudaGetLastError());
}
