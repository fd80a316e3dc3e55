// Operand validation with the reference provider's rules and error codes
// (src/sparse/cuda/operations.cc:22-398).  Everything here runs on the host
// before any work is enqueued, so a failing call never mutates an output.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../../include/asc_sparse_b200.h"

namespace ascb::host {

struct Status {
  int code = ASC_SB_OK;
  std::string message;
  bool ok() const { return code == ASC_SB_OK; }
  static Status Ok() { return {}; }
};

inline Status Fail(int code, const char* message) { return {code, message}; }

struct Span {
  const void* begin = nullptr;
  std::size_t bytes = 0;
};

struct SparseBytes {
  std::size_t first = 0;   // outer offsets
  std::size_t second = 0;  // inner indices
  std::size_t values = 0;
};

std::size_t ElementBytes(int kind);
bool Overlap(Span a, Span b);

// ValidateSparseMetadata + ValidateSparseDevice (operations.cc:134-276).
Status ValidateSparse(const asc_sb_sparse& m, int device, SparseBytes* bytes);
// The metadata half alone (format, kind, extents, trust, sizes, alignment,
// overlap): no memory-space or pointer-attribute checks.
Status ValidateSparseMetadata(const asc_sb_sparse& m, SparseBytes* bytes);
// VectorBytes + ValidateVector (operations.cc:278-332).  `span` receives the
// bytes actually touched by the vector (lowest to highest element).
Status ValidateVector(const asc_sb_vector& v, int kind, bool writable,
                      int device, Span* span);
// ValidateMatrixDevice (operations.cc:609-679).
Status ValidateDense(const asc_sb_dense& d, int kind, bool writable,
                     int device, Span* span);
// Device pointer check via cudaPointerGetAttributes (operations.cc:109-128).
Status ValidateDevicePointer(const void* p, std::size_t bytes, int device,
                             const char* message);
Status ValidateAddress(const void* p, std::size_t bytes, std::size_t alignment,
                       const char* null_message, const char* align_message);

}  // namespace ascb::host
