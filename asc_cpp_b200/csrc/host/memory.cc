#include "memory.h"

#include <cuda_runtime.h>

namespace ascb::host {

bool Acquire(const Allocator& allocator, std::size_t bytes, int space, Block* out) {
  *out = Block{};
  void* p = nullptr;
  if (allocator.allocate != nullptr) {
    p = allocator.allocate(allocator.user, bytes, space);
  } else {
    const cudaError_t e = space == ASC_SB_PINNED_HOST
                              ? cudaHostAlloc(&p, bytes, cudaHostAllocDefault)
                              : cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
    }
  }
  if (p == nullptr) return false;
  *out = Block{p, bytes, space, allocator};
  return true;
}

void Release(Block* block) {
  if (block->ptr == nullptr) return;
  if (block->from.release != nullptr) {
    block->from.release(block->from.user, block->ptr, block->bytes, block->space);
  } else if (block->from.allocate == nullptr) {
    if (block->space == ASC_SB_PINNED_HOST) {
      (void)cudaFreeHost(block->ptr);
    } else {
      (void)cudaFree(block->ptr);
    }
  }
  *block = Block{};
}

}  // namespace ascb::host
