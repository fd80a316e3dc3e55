// Read access to a context's fields for entry points defined outside api.cc.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../../include/asc_sparse_b200.h"
#include "memory.h"

namespace ascb::host {

struct ContextView {
  int device = 0;
  cudaStream_t stream = nullptr;
  int determinism = ASC_SB_DETERMINISTIC;
  int sm_count = 148;
  std::mutex* mutex = nullptr;
  std::string* last_error = nullptr;
  std::atomic<std::int64_t>* launches = nullptr;
  void** stager = nullptr;  // clone staging (clone.cc), created on first use
  const Allocator* allocator = nullptr;  // for the context's own memory
};

// False for a null context.
bool ViewContext(asc_sb_context* context, ContextView* view);
// Releases a context's clone staging (pinned buffers, copy threads).
void DestroyStager(void* stager);

}  // namespace ascb::host
