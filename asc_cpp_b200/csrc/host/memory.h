// Memory a context allocates for itself after creation (solve scratch,
// selector parameters, clone staging), through the caller's allocator when
// one is installed (asc_sb_context_set_allocator), else cudaMalloc /
// cudaHostAlloc.  Each block remembers the allocator that gave it, so it goes
// back there even if the context's allocator changes meanwhile.
#pragma once

#include <cstddef>

#include "../../../include/asc_sparse_b200.h"

namespace ascb::host {

struct Allocator {
  asc_sb_allocate_fn allocate = nullptr;  // nullptr: the CUDA runtime
  asc_sb_deallocate_fn release = nullptr;
  void* user = nullptr;
};

struct Block {
  void* ptr = nullptr;
  std::size_t bytes = 0;
  int space = ASC_SB_DEVICE;  // ASC_SB_DEVICE or ASC_SB_PINNED_HOST
  Allocator from;
};

// Allocates `bytes` in `space` (ASC_SB_DEVICE or ASC_SB_PINNED_HOST); false on
// failure, with `out` left empty.
bool Acquire(const Allocator& allocator, std::size_t bytes, int space, Block* out);
// Returns a block to the allocator that gave it (no-op for an empty block).
void Release(Block* block);

}  // namespace ascb::host
