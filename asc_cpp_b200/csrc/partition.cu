// Partition kernels: integer-only, bit-exact.  Each thread places one tile
// boundary by binary search over the CSR row offsets.
#include "common.cuh"
#include "kernels.h"

namespace ascb {
namespace {

constexpr int kPartitionThreads = 256;

// Tile k starts at the first row r with weight*r + ptr[r] >= k*items; the
// last bound is `rows`.
__global__ void __launch_bounds__(kPartitionThreads)
row_tile_kernel(int64_t rows, const int64_t* __restrict__ ptr, int64_t items, int64_t weight,
                int64_t* __restrict__ tile_row, int64_t ntiles) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k > ntiles) return;
  tile_row[k] = k == ntiles ? rows : first_row_at(ptr, rows, weight, k * items);
}

// Merge-path split of diagonal d: the first i in [max(0, d-nnz), min(d, rows)]
// with ptr[i+1] > d - i - 1 (row ends merged against nonzero positions).
__global__ void __launch_bounds__(kPartitionThreads)
merge_split_kernel(int64_t rows, const int64_t* __restrict__ ptr, int64_t nnz,
                   int64_t items, int64_t* __restrict__ split_row,
                   int64_t* __restrict__ split_nz, int64_t ntiles) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k > ntiles) return;
  const int64_t total = rows + nnz;
  const int64_t d = k * items < total ? k * items : total;
  int64_t lo = d - nnz > 0 ? d - nnz : 0;
  int64_t hi = d < rows ? d : rows;
  while (lo < hi) {
    const int64_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(ptr + mid + 1) <= d - mid - 1) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  split_row[k] = lo;
  split_nz[k] = d - lo;
}

unsigned blocks_for(int64_t threads) {
  return static_cast<unsigned>((threads + kPartitionThreads - 1) / kPartitionThreads);
}

}  // namespace
}  // namespace ascb

extern "C" {

int64_t ascb_row_tile_count(int64_t rows, int64_t nnz, int64_t items, int64_t weight) {
  if (rows <= 0) return 0;
  return (weight * rows + nnz + items - 1) / items;
}

int ascb_row_tiles(void* stream, const ascb_csr* a, int64_t items, int64_t weight,
                   int64_t* tile_row, int64_t ntiles) {
  if (ntiles <= 0) return 0;
  ascb::row_tile_kernel<<<ascb::blocks_for(ntiles + 1), ascb::kPartitionThreads, 0,
                          static_cast<cudaStream_t>(stream)>>>(a->rows, a->ptr, items, weight,
                                                               tile_row, ntiles);
  return static_cast<int>(cudaGetLastError());
}

int64_t ascb_merge_tile_count(int64_t rows, int64_t nnz, int64_t items) {
  if (rows <= 0) return 0;
  return (rows + nnz + items - 1) / items;
}

int ascb_merge_path_splits(void* stream, const ascb_csr* a, int64_t items,
                           int64_t* split_row, int64_t* split_nz, int64_t ntiles) {
  if (ntiles <= 0) return 0;
  ascb::merge_split_kernel<<<ascb::blocks_for(ntiles + 1), ascb::kPartitionThreads, 0,
                             static_cast<cudaStream_t>(stream)>>>(
      a->rows, a->ptr, a->nnz, items, split_row, split_nz, ntiles);
  return static_cast<int>(cudaGetLastError());
}

}  // extern "C"
