/*
 * asc_sparse_b200.h - C ABI of the B200-native Sparse BLAS hot path.
 *
 * This library replaces the computational back end of ASCCpp's experimental
 * `sparse_cuda` provider facet (reference: include/asc/sparse/providers/
 * cuda.h, src/sparse/cuda/operations.cc, src/sparse/cuda/kernels.cu).  Every
 * entry point takes plain pointers, sizes and enums -- no C++ or torch types --
 * so that the reference's exported `internal_sparse_cuda::*Erased` functions
 * can forward to it one-for-one (asc_cpp_b200/binding/sparse_cuda_provider.cc
 * is that forwarding layer), and so that ctypes, cgo or any other FFI can
 * bind it directly.
 *
 * Semantics mirror the reference exactly:
 *   - enum values are numerically identical to the reference enums;
 *   - status codes are the reference's asc::ErrorCode values
 *     (include/asc/core/status.h:35-55);
 *   - every call validates completely before it enqueues anything, so a
 *     failing call never writes an output (operations.cc:349-398);
 *   - work is enqueued on the context's stream; success never implies a host
 *     wait (docs/modules/sparse.md:441-442);
 *   - a failure detected after enqueue synchronizes the stream before it
 *     returns (operations.cc:1027-1045).
 * All kernels are hand-written for sm_100a; there is no cuSPARSE, cuBLAS or
 * CPU fallback behind any entry point.
 */
#ifndef ASC_SPARSE_B200_H_
#define ASC_SPARSE_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define ASC_SB_API __declspec(dllexport)
#else
#define ASC_SB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums (values identical to the reference) --------------------------- */

/* asc::ErrorCode, include/asc/core/status.h:35-55 */
typedef enum asc_sb_status {
  ASC_SB_OK = 0,
  ASC_SB_INVALID_ARGUMENT = 1,
  ASC_SB_SHAPE = 2,
  ASC_SB_INDEX = 3,
  ASC_SB_OVERFLOW = 4,
  ASC_SB_INVALID_STATE = 5,
  ASC_SB_ALLOCATION = 6,
  ASC_SB_MEMORY_ACCESS = 7,
  ASC_SB_MEMORY_TRANSFER = 8,
  ASC_SB_UNSUPPORTED = 9,
  ASC_SB_UNAVAILABLE = 10,
  ASC_SB_PROVIDER = 11,
  ASC_SB_NUMERICAL = 12,
  ASC_SB_INTERNAL = 18
} asc_sb_status;

/* asc::MemorySpace, include/asc/core/memory.h:30-35 */
enum { ASC_SB_HOST = 0, ASC_SB_PINNED_HOST = 1, ASC_SB_DEVICE = 2,
       ASC_SB_MANAGED = 3 };

/* internal_sparse_cuda::ElementKind, include/asc/sparse/providers/cuda.h:103-108 */
enum { ASC_SB_FLOAT = 0, ASC_SB_DOUBLE = 1, ASC_SB_COMPLEX_FLOAT = 2,
       ASC_SB_COMPLEX_DOUBLE = 3 };

/* internal_sparse_cuda::FormatKind, cuda.h:123-127 */
enum { ASC_SB_COORDINATE = 0, ASC_SB_CSR = 1, ASC_SB_CSC = 2 };

/* asc::SparseBlasTranspose, include/asc/sparse/blas.h:88-92 */
enum { ASC_SB_OP_NONE = 0, ASC_SB_OP_TRANSPOSE = 1,
       ASC_SB_OP_CONJUGATE_TRANSPOSE = 2 };

/* asc::SparseBlasLayout, include/asc/sparse/blas.h:103-106 */
enum { ASC_SB_COLUMN_MAJOR = 0, ASC_SB_ROW_MAJOR = 1 };

/* asc::Determinism, include/asc/core/execution.h:122-125.  DETERMINISTIC (the
 * reference's default) runs the row-ordered kernels, which reproduce the
 * reference's serial summation order and rounding bit for bit.
 * BACKEND_DEFAULT lets the library pick the fastest variant, whose results
 * stay within |y - y_ref| <= gamma_{n+2} * (|alpha| |A| |x| + |beta| |y|),
 * gamma_k = k u / (1 - k u), n = stored entries of the row. */
enum { ASC_SB_DETERMINISTIC = 0, ASC_SB_BACKEND_DEFAULT = 1 };

/* SpMV kernel variants (no reference counterpart; the reference has one
 * thread-per-row kernel, src/sparse/cuda/kernels.cu:91-115). */
enum {
  ASC_SB_VARIANT_AUTO = -1,       /* library choice (selector / heuristics)   */
  ASC_SB_VARIANT_ROW_ORDERED = 0, /* warp row tiles, bit-exact serial order   */
  ASC_SB_VARIANT_VECTOR = 1,      /* 'lanes' threads per row, shuffle sums    */
  ASC_SB_VARIANT_WARP_TILES = 2,  /* warp row tiles, FMA, parallel long rows  */
  ASC_SB_VARIANT_MERGE_PATH = 3,  /* merge-path partition (one item per row
                                     and per nonzero) on the register-
                                     segmented tile body; unaligned arrays:
                                     the warp kernel                          */
  ASC_SB_VARIANT_ROW_SPLIT = 4    /* warp row tiles; long rows' tails split
                                     into 256-entry chunks over many warps   */
};

/* ---- descriptors ---------------------------------------------------------- */

/* internal_sparse_cuda::SparseDescriptor, cuda.h:143-156 (rank fixed at two).
 * CSR: structure_first = int64 outer offsets [rows+1],
 *      structure_second = int64 column indices [nonzeros].
 * CSC: outer offsets over columns [columns+1], row indices [nonzeros].
 * Structure must be canonical (zero based, sorted, unique) and the caller
 * asserts that by setting canonical_structure_trusted, exactly as the
 * reference's trusted device clones do (compressed.h:759-770). */
typedef struct asc_sb_sparse {
  const void* structure_first;
  const void* structure_second;
  const void* values;
  int32_t memory_space;
  int32_t element_kind;
  int32_t format;
  int32_t canonical_structure_trusted;
  int64_t rows;
  int64_t columns;
  int64_t nonzeros;
} asc_sb_sparse;

/* internal_sparse_cuda::VectorDescriptor, cuda.h:164-173.  Element i is at
 * data[i * stride]; for a negative stride `data` is logical element 0 and
 * reachable_data/reachable_size (optional) give the backing span. */
typedef struct asc_sb_vector {
  const void* data;
  const void* reachable_data;
  size_t reachable_size;
  int32_t memory_space;
  int32_t element_kind;
  int64_t extent;
  int64_t stride;
  int32_t writable;
  int32_t reserved;
} asc_sb_vector;

/* internal_sparse_cuda::MatrixDescriptor, cuda.h:186-197. */
typedef struct asc_sb_dense {
  const void* data;
  const void* reachable_data;
  size_t reachable_size;
  int32_t memory_space;
  int32_t element_kind;
  int64_t rows;
  int64_t columns;
  int64_t leading_dimension;
  int32_t layout;
  int32_t writable;
} asc_sb_dense;

typedef struct asc_sb_context asc_sb_context;

/* ---- context -------------------------------------------------------------- */

/* Replaces SparseCudaContext::Create (cuda.h:514; src/sparse/cuda/context.cc:
 * 69-113).  `stream` is a cudaStream_t on `device` (the reference passes the
 * ExecutionContext's native stream, src/core/cuda/runtime.cc:454; the legacy
 * default stream is cudaStreamLegacy, (void*)0x1); NULL makes the context
 * create and own a non-blocking stream.  Determinism starts at
 * ASC_SB_DETERMINISTIC, the reference default (execution.h:162). */
ASC_SB_API int asc_sb_context_create(int32_t device, void* stream,
                                     asc_sb_context** out);
/* Replaces ~SparseCudaContext (cuda.h:588). NULL is accepted. */
ASC_SB_API int asc_sb_context_destroy(asc_sb_context* context);
ASC_SB_API int asc_sb_context_set_determinism(asc_sb_context* context,
                                              int32_t determinism);
/* Forces one SpMV variant (for autotuning and tests); BACKEND_DEFAULT only
 * (DETERMINISTIC always runs the bit-exact kernels).  `lanes` (1..32, power
 * of two; 0 = auto) is the threads per row of VECTOR, and for ROW_SPLIT the
 * number of 256-entry rounds a row may run past its tile before its tail is
 * split over other warps (0 = 4).  ROW_SPLIT needs a plan or the
 * asc_sb_csr_spmv workspace for its chunk table; without one (the standard
 * path without a plan) long rows run inline as in WARP_TILES.  Its partial
 * sums are combined in a fixed order, so results repeat run to run. */
ASC_SB_API int asc_sb_context_set_variant(asc_sb_context* context,
                                          int32_t variant, int32_t lanes);
/* Allocator for the memory a context allocates for itself after creation:
 * the scratch of triangular solves without a plan (device; it grows to the
 * largest solve), the variant selector's parameters (device) and the clone
 * staging buffers (pinned host).  `allocate` returns NULL on failure; the
 * call that needed the memory then returns ASC_SB_ALLOCATION without having
 * touched its outputs, and the context stays usable.  `release` (may be
 * NULL: blocks are then never returned) gets back every block `allocate`
 * gave, with the same size and space, when the context no longer needs it.
 * Passing NULL for `allocate` restores cudaMalloc / cudaHostAlloc.  Lets a
 * host application that owns all device memory, or a test that fails chosen
 * allocations, serve these requests.  No counterpart in the reference (its
 * provider allocates only from the caller's MemoryResource, in clones). */
typedef void* (*asc_sb_allocate_fn)(void* user, size_t bytes, int32_t memory_space);
typedef void (*asc_sb_deallocate_fn)(void* user, void* pointer, size_t bytes,
                                     int32_t memory_space);
ASC_SB_API int asc_sb_context_set_allocator(asc_sb_context* context,
                                            asc_sb_allocate_fn allocate,
                                            asc_sb_deallocate_fn release, void* user);
/* Longest time a kernel of this context spins on a value another warp has
 * not published yet (the dependencies of triangular solves) before it gives
 * up: the call's results are then invalid, the device status word
 * (asc_sb_context_device_status) becomes 1, every other wait of the launch
 * ends at once, and the kernel returns, leaving the context usable.
 * 0 restores the default, 2 s.  No counterpart in the reference. */
ASC_SB_API int asc_sb_context_set_wait_limit(asc_sb_context* context,
                                             int64_t nanoseconds);
ASC_SB_API void* asc_sb_context_stream(const asc_sb_context* context);
ASC_SB_API int asc_sb_context_synchronize(asc_sb_context* context);
/* Message of the most recent failure on this context ("" if none). */
ASC_SB_API const char* asc_sb_context_last_error(const asc_sb_context* context);
/* Kernel launches issued by this context since creation (instrumentation). */
ASC_SB_API int64_t asc_sb_context_launch_count(const asc_sb_context* context);
/* Reads (and optionally clears) the context's device status word: nonzero
 * means a kernel gave up a bounded wait and its results are not valid.
 * Synchronizes the context stream. */
ASC_SB_API int asc_sb_context_device_status(asc_sb_context* context,
                                            int32_t* value, int32_t clear);

/* ---- compat SpMV  y = alpha * A * x + beta * y ----------------------------- */

/* Replaces internal_sparse_cuda::CsrSpmvWorkspaceSizeErased (cuda.h:220-222;
 * operations.cc:884-909).  The size is stable for a given (A, x, y) shape. */
ASC_SB_API int asc_sb_csr_spmv_workspace_size(asc_sb_context* context,
                                              const asc_sb_sparse* matrix,
                                              const asc_sb_vector* input,
                                              const asc_sb_vector* output,
                                              size_t* bytes);

/* Replaces internal_sparse_cuda::CsrSpmvErased (cuda.h:224-227;
 * operations.cc:911-1049) and the compat path it serves
 * (SpmvReferenceImpl, src/sparse/reference_blas.cc:9-41).  alpha and beta
 * arrive as double for both element kinds and are rounded to the element type
 * (operations.cc:1010-1013).  beta == 0 never reads y.  `workspace` must be
 * device memory of at least the queried size (or NULL/0 when that size is 0),
 * 256-byte aligned and disjoint from every operand. */
ASC_SB_API int asc_sb_csr_spmv(asc_sb_context* context, double alpha,
                               const asc_sb_sparse* matrix,
                               const asc_sb_vector* input, double beta,
                               const asc_sb_vector* output, void* workspace,
                               size_t workspace_bytes,
                               int32_t workspace_space);

/* Compat SpMV that allocates nothing and takes no workspace.  No counterpart
 * in the reference.  It is for callers that cannot allocate device memory
 * when they need the product and cannot hand in a workspace either: plugin
 * hosts whose device memory belongs to the host application's own allocator,
 * which forbids raw device allocations by plugins, and latency-critical loops
 * that must not risk the implicit device synchronisation of cudaMalloc or
 * cudaFree.  Same validation, error codes and arithmetic as asc_sb_csr_spmv
 * with the context's determinism; it always runs the default kernel,
 * ignoring a variant forced with asc_sb_context_set_variant or picked by the
 * selector.  In DETERMINISTIC mode its results equal asc_sb_csr_spmv's bit
 * for bit; in BACKEND_DEFAULT mode both meet the same error bound and are
 * equal whenever asc_sb_csr_spmv also runs the default kernel.  Its only
 * scratch, the row-tile partition, is a static 2 MiB device array per GPU
 * (held from library load until process exit): matrices needing more than
 * 262,144 tile bounds -- ceil((2*rows + nnz)/251) + 1 when the index and
 * value arrays start on 16-byte boundaries, ceil((8*rows + nnz)/256) + 1
 * otherwise -- are rejected with ASC_SB_UNSUPPORTED.  All calls on a device share that array: calls that
 * overlap on the GPU race.  The first call on each device looks up the
 * array's device address, once; make that first call before any stream
 * capture starts on the device.  A cudaDeviceReset invalidates the address
 * looked up; do not use this entry point after one in the same process. */
ASC_SB_API int asc_sb_csr_spmv_no_alloc(asc_sb_context* context, double alpha,
                                        const asc_sb_sparse* matrix,
                                        const asc_sb_vector* input, double beta,
                                        const asc_sb_vector* output);

/* ---- standard SpMV / SpMM  y += alpha * op(A) * x -------------------------- */

/* Replaces internal_sparse_cuda::StandardSpmvErased (cuda.h:243-246;
 * operations.cc:1214-1299) and the CPU template it must agree with
 * (blas.h:1607-1667).  alpha_imag must be 0 (real element kinds).  CSR and
 * CSC are both accepted: CSC with op = none is computed as the transpose of
 * the CSR matrix with the same arrays.  A transpose (of CSR) in
 * DETERMINISTIC mode runs on the transposed structure: a plan's
 * (asc_sb_plan_create with ASC_SB_PLAN_TRANSPOSE), or, without a plan, one
 * rebuilt for the call in the context's scratch buffer (which grows, after a
 * stream drain, from the context's allocator).  BACKEND_DEFAULT without a
 * plan scatters with atomics. */
ASC_SB_API int asc_sb_standard_spmv(asc_sb_context* context, int32_t op,
                                    double alpha_real, double alpha_imag,
                                    const asc_sb_sparse* matrix,
                                    const asc_sb_vector* input,
                                    const asc_sb_vector* output);

/* Replaces internal_sparse_cuda::StandardSpmmErased (cuda.h:248-251;
 * operations.cc:1301-1378), CPU contract blas.h:1692-1750. */
ASC_SB_API int asc_sb_standard_spmm(asc_sb_context* context, int32_t op,
                                    double alpha_real, double alpha_imag,
                                    const asc_sb_sparse* matrix,
                                    const asc_sb_dense* input,
                                    const asc_sb_dense* output);

/* ---- Level-1 on an indexed vector ------------------------------------------ */

/* internal_sparse_cuda::IndexedVectorDescriptor, cuda.h:175-184: int64
 * indices [nonzeros] (sorted, unique, below dense_extent; the caller asserts
 * it with canonical_structure_trusted) and values [nonzeros]. */
typedef struct asc_sb_indexed_vector {
  const void* indices;
  const void* values;
  int32_t memory_space;
  int32_t element_kind;
  int64_t nonzeros;
  int64_t dense_extent;
  int32_t writable;
  int32_t canonical_structure_trusted;
} asc_sb_indexed_vector;

/* internal_sparse_cuda::StandardOperation, cuda.h:111-117 */
enum { ASC_SB_L1_DOT = 0, ASC_SB_L1_AXPY = 1, ASC_SB_L1_GATHER = 2,
       ASC_SB_L1_GATHER_ZERO = 3, ASC_SB_L1_SCATTER = 4 };
/* asc::SparseBlasConjugation, blas.h:74-77 */
enum { ASC_SB_UNCONJUGATED = 0, ASC_SB_CONJUGATED = 1 };

/* Replaces internal_sparse_cuda::StandardLevel1Erased (cuda.h:234-238;
 * operations.cc:1122-1212), CPU contract blas.h:1340-1600:
 *   DOT          result[0] = sum_k v'_k x[i_k]  (v' = conj(v) if CONJUGATED)
 *   AXPY         x[i_k] += alpha v_k   (alpha == 0: nothing is touched)
 *   GATHER       v_k = x[i_k]
 *   GATHER_ZERO  v_k = x[i_k]; x[i_k] = 0
 *   SCATTER      x[i_k] = v_k
 * All four element kinds.  The element-wise operations are exact; the dot in
 * DETERMINISTIC mode adds in stored order with the reference's rounding (bit
 * for bit), in BACKEND_DEFAULT mode with a fixed reduction tree. */
ASC_SB_API int asc_sb_standard_level1(asc_sb_context* context, int32_t operation,
                                      int32_t conjugation, double alpha_real,
                                      double alpha_imag,
                                      const asc_sb_indexed_vector* sparse,
                                      const asc_sb_vector* dense,
                                      const asc_sb_vector* result);

/* asc::SparseBlasTriangle / SparseBlasDiagonal, blas.h:117-134 */
enum { ASC_SB_UPPER = 0, ASC_SB_LOWER = 1 };
enum { ASC_SB_NON_UNIT = 0, ASC_SB_UNIT = 1 };

/* Replaces internal_sparse_cuda::StandardTriangularSolveErased (cuda.h:250-253;
 * operations.cc:1380-1451), behind CudaSparseTriangularSolve[Multiple]
 * (cuda.h:1680-1739); CPU contract blas.h:1774-1910.  Solves
 * op(A) X = alpha B in place for the square CSR matrix A and the n x k dense
 * right-hand sides (a vector is n x 1 row major with the increment as leading
 * dimension).  triangle names A's triangle; entries of the other strict
 * triangle are ignored; with ASC_SB_NON_UNIT the stored diagonal divides (a
 * missing one divides by zero).  alpha == 0 writes zeros without reading B.
 * DETERMINISTIC: the reference's order and rounding, bit for bit (complex
 * division by Smith's method as the facet's kernel does); BACKEND_DEFAULT:
 * contracted sums within gamma_{m+2} of the row's terms.  One launch, sync
 * free, waits bounded (asc_sb_context_device_status reads 1 if one gave up).  The ready
 * flags live in a context-owned buffer that grows to the largest n (and, for
 * op != none, also holds the transposed structure, rebuilt per call); use a
 * plan to keep all memory caller-provided. */
ASC_SB_API int asc_sb_standard_triangular_solve(asc_sb_context* context, int32_t op,
                                                double alpha_real, double alpha_imag,
                                                const asc_sb_sparse* matrix,
                                                int32_t triangle, int32_t diagonal,
                                                const asc_sb_dense* right_hand_sides);

/* ---- host -> device clones ------------------------------------------------
 * Replace the copy half of internal_sparse_cuda::CloneCsrErased and
 * CloneIndexedErased (cuda.h:212-219; operations.cc:696-880).  The caller
 * allocates the destination arrays (in the reference the clone allocates them
 * from the caller's MemoryResource) and describes them with the source's
 * shape, kind and nonzero count in device memory.  The copies are enqueued on
 * the context stream.  Pageable sources (ASC_SB_HOST) are staged through a
 * context-owned pinned ring filled by host copy threads (created on first
 * use): when the call returns, the source has been read completely.
 * Page-locked sources are copied by DMA directly and must stay unchanged
 * until the stream has passed the copy.  The source must be canonical
 * (canonical_structure_trusted, as the reference's host views guarantee);
 * the destination is then a trusted device array. */
ASC_SB_API int asc_sb_clone_csr(asc_sb_context* context, const asc_sb_sparse* source,
                                const asc_sb_sparse* destination);
ASC_SB_API int asc_sb_clone_indexed(asc_sb_context* context,
                                    const asc_sb_indexed_vector* source,
                                    const asc_sb_indexed_vector* destination);

/* ---- analysis plans (no reference counterpart) ----------------------------
 * A plan caches, in caller-provided device memory, everything the kernels can
 * reuse across calls on one matrix: the row-tile and merge-path partitions and
 * (optionally) the transposed structure with its values.  The matrix's values
 * must not change while a plan built with ASC_SB_PLAN_TRANSPOSE is in use
 * (call asc_sb_plan_refresh_values after changing them). */
/* ASC_SB_PLAN_TRIANGULAR adds the ready flags of triangular solves
 * (asc_sb_plan_triangular_solve); solves through one plan must be ordered
 * (one stream). */
/* ASC_SB_PLAN_ROW_GROUPS (CSR, float or double) prepares two more SpMM
 * kernels for asc_sb_plan_standard_spmm with op = none and row-major B and C
 * whose rows are whole 16-byte chunks on 16-byte boundaries:
 *   - the TMA-staged kernel: per group of 16, 32 or 64 rows (three levels;
 *     asc_sb_plan_spmm_stage_rows), the distinct columns in runs of
 *     consecutive columns and per stored entry the slot of its column; a
 *     producer warp per CTA stages a stage's rows of B, row offsets, values,
 *     slots (and long rows of C) in shared memory with bulk copies
 *     (two-stage pipeline) and the other warps compute from there.  By
 *     default it runs when the groups share columns (at least 1.25 entries
 *     per distinct column of a 16-row group), k >= 8 and two stages fit one
 *     CTA's shared memory;
 *   - row groups of R rows (R = 8 at creation): runs -- one per distinct
 *     column, with the rows that hold it -- so that each row of B is loaded
 *     once per run and applied to all of the run's rows.  Used only when
 *     chosen: by asc_sb_plan_spmm_autotune or asc_sb_plan_set_spmm.
 * Every kernel adds each row's entries in stored order: DETERMINISTIC results
 * stay bit-identical to the reference. */
enum { ASC_SB_PLAN_TRANSPOSE = 1, ASC_SB_PLAN_TRIANGULAR = 2, ASC_SB_PLAN_ROW_GROUPS = 4 };
typedef struct asc_sb_plan asc_sb_plan;
ASC_SB_API int asc_sb_plan_workspace_size(asc_sb_context* context,
                                          const asc_sb_sparse* matrix,
                                          int32_t flags, size_t* bytes);
ASC_SB_API int asc_sb_plan_create(asc_sb_context* context,
                                  const asc_sb_sparse* matrix, int32_t flags,
                                  void* workspace, size_t workspace_bytes,
                                  asc_sb_plan** out);
ASC_SB_API int asc_sb_plan_refresh_values(asc_sb_context* context,
                                          asc_sb_plan* plan);
ASC_SB_API int asc_sb_plan_destroy(asc_sb_plan* plan);
/* Compat SpMV through a plan: same contract as asc_sb_csr_spmv. */
ASC_SB_API int asc_sb_plan_csr_spmv(asc_sb_context* context,
                                    const asc_sb_plan* plan, double alpha,
                                    const asc_sb_vector* input, double beta,
                                    const asc_sb_vector* output);
/* Standard SpMV through a plan: same contract as asc_sb_standard_spmv.  With
 * ASC_SB_PLAN_TRANSPOSE, a transposed product (op != none on CSR, op = none
 * on CSC) runs the stored-order kernels on the transposed structure, so it is
 * available in DETERMINISTIC mode and reproduces the reference's order
 * (blas.h:1241-1256: outer then inner) bit for bit. */
ASC_SB_API int asc_sb_plan_standard_spmv(asc_sb_context* context,
                                         const asc_sb_plan* plan, int32_t op,
                                         double alpha_real, double alpha_imag,
                                         const asc_sb_vector* input,
                                         const asc_sb_vector* output);
/* What a plan found and holds (bit set): the transposed structure, and
 * dense, aligned 16 x 16 blocks in an FP32 CSR matrix.  For the latter,
 * asc_sb_plan_standard_spmm with op = none, row-major B and C, in
 * BACKEND_DEFAULT mode with variant AUTO, runs on the tensor cores (tcgen05,
 * FP32 operands split into three TF32 products), within
 * |c - c_exact| <= (n + 64) 2^-22 |alpha| sum_k |a_k b_k| + 2^-23 |c0| per
 * output (n = stored entries of the row). */
enum { ASC_SB_PLAN_HAS_TRANSPOSE = 1, ASC_SB_PLAN_HAS_BLOCKS16 = 2,
       ASC_SB_PLAN_HAS_ROW_GROUPS = 4 /* SpMM runs through the row groups */,
       ASC_SB_PLAN_HAS_STAGED_SPMM = 8 /* SpMM runs through the staged kernel */ };
ASC_SB_API int asc_sb_plan_properties(const asc_sb_plan* plan,
                                      int32_t* properties);
/* Standard SpMM through a plan: same contract as asc_sb_standard_spmm, with
 * the transposed products of asc_sb_plan_standard_spmv and the tensor-core
 * path for dense 16 x 16 blocks above. */
ASC_SB_API int asc_sb_plan_standard_spmm(asc_sb_context* context,
                                         const asc_sb_plan* plan, int32_t op,
                                         double alpha_real, double alpha_imag,
                                         const asc_sb_dense* input,
                                         const asc_sb_dense* output);
/* SpMM autotuner of a plan created with ASC_SB_PLAN_ROW_GROUPS: times, on
 * these operands (C += alpha * A * B, `reps` products each plus one warm-up,
 * CUDA events on the context stream), the row-by-row kernel, the TMA-staged
 * kernel (where it fits) and the row-group kernel with R = 2, 4, 8, 16 and 32
 * rows per group (k-tile and lanes per row follow from R and k), keeps the
 * fastest for the plan's later products and returns its time per product and
 * R (0: row by row; ASC_SB_SPMM_STAGED: the staged kernel).  The products run
 * for real, so C accumulates.  No counterpart in the reference. */
enum { ASC_SB_SPMM_STAGED = -1, ASC_SB_SPMM_AUTO = -2 };
/* Chooses the SpMM kernel of a plan created with ASC_SB_PLAN_ROW_GROUPS:
 * 0 = row by row, ASC_SB_SPMM_STAGED = the TMA-staged kernel wherever it fits
 * (any k), R = 2, 4, 8, 16 or 32 = row groups of R rows (rebuilt on the
 * stream), ASC_SB_SPMM_AUTO = the defaults above. */
ASC_SB_API int asc_sb_plan_set_spmm(asc_sb_context* context, asc_sb_plan* plan,
                                    int32_t choice);
ASC_SB_API int asc_sb_plan_spmm_autotune(asc_sb_context* context,
                                         asc_sb_plan* plan, double alpha,
                                         const asc_sb_dense* input,
                                         const asc_sb_dense* output, int32_t reps,
                                         float* best_ms, int32_t* rows_per_group);
/* Rows per group of the staged SpMM tables a product with k columns of
 * row-major B and C (leading dimension k) would run on: 16, 32 or 64 (wide
 * groups of two or four 16-row groups, one slot per distinct column) -- of
 * the levels whose two stages fit a CTA's shared memory, the one that keeps
 * the most CTAs per SM, the widest among equals -- or 0 where the staged
 * kernel does not apply (no staged tables, element kind or k unsupported, or
 * no stage fits).  Whether the staged kernel runs at all is the plan's SpMM
 * choice (ASC_SB_PLAN_HAS_STAGED_SPMM, asc_sb_plan_set_spmm). */
ASC_SB_API int asc_sb_plan_spmm_stage_rows(asc_sb_context* context, const asc_sb_plan* plan,
                                           int64_t k, int64_t* rows);
/* The last asc_sb_plan_spmm_autotune's table: *count candidates in the order
 * timed (R as returned by the autotuner) and their ms per product; up to
 * `capacity` of them are copied. */
ASC_SB_API int asc_sb_plan_spmm_tuning(const asc_sb_plan* plan, int32_t capacity,
                                       int32_t* count, int32_t* candidates, float* ms);

/* Triangular solve through a plan created with ASC_SB_PLAN_TRIANGULAR: same
 * contract as asc_sb_standard_triangular_solve on the plan's matrix; op !=
 * none also needs ASC_SB_PLAN_TRANSPOSE (else ASC_SB_INVALID_STATE) and reuses
 * the plan's transposed structure.  Allocates nothing.  After
 * asc_sb_plan_triangular_analysis for the same op class (none / transposed)
 * and triangle, rows are scheduled in dependency-level order, which keeps
 * wide wavefronts (e.g. grid stencils) in flight at once; the arithmetic and
 * its results are unchanged. */
ASC_SB_API int asc_sb_plan_triangular_analysis(asc_sb_context* context,
                                               asc_sb_plan* plan, int32_t op,
                                               int32_t triangle);
ASC_SB_API int asc_sb_plan_triangular_solve(asc_sb_context* context,
                                            const asc_sb_plan* plan, int32_t op,
                                            double alpha_real, double alpha_imag,
                                            int32_t triangle, int32_t diagonal,
                                            const asc_sb_dense* right_hand_sides);

/* ---- format conversion on the device --------------------------------------
 * Stable conversions of device data, bit-identical to the reference's host
 * conversions: entries land in the destination grouped by their new outer
 * index and, within one outer index, in source storage order.  The
 * destination descriptor names caller-allocated device arrays of the target
 * format (offsets [outer + 1], indices [nonzeros], values [nonzeros]) with the
 * source's element kind and shape; they are written on the context stream.
 * The workspace is device memory, 256-byte aligned, of the queried size; it
 * may be reused once the stream has passed the call. */
ASC_SB_API int asc_sb_convert_workspace_size(asc_sb_context* context,
                                             int64_t rows, int64_t columns,
                                             int64_t nonzeros,
                                             int32_t destination_format,
                                             size_t* bytes);
/* CSR -> CSC or CSC -> CSR.  Replaces, for device data, asc::ConvertToCsc(
 * CsrView) and asc::ConvertToCsr(CscView) (include/asc/sparse/compressed.h:
 * 1728-1780 -> CompressedSparseArray::FromCompressed, :1151-1221). */
ASC_SB_API int asc_sb_convert_compressed(asc_sb_context* context,
                                         const asc_sb_sparse* source,
                                         const asc_sb_sparse* destination,
                                         void* workspace,
                                         size_t workspace_bytes);
/* Coordinates -> CSR or CSC.  `coordinates` holds (row, column) int64 pairs,
 * [nonzeros][2], the reference's coordinate storage (coordinate.h:267-330);
 * `values` holds `nonzeros` elements of `element_kind`.  Replaces, for device
 * data, asc::ConvertToCsr / ConvertToCsc(CoordinateView) (compressed.h:
 * 1676-1726 -> CompressedSparseArray::FromCoordinate, :1082-1131).  Input in
 * any order is accepted; canonical input gives canonical output. */
ASC_SB_API int asc_sb_convert_coordinates(asc_sb_context* context,
                                          const int64_t* coordinates,
                                          const void* values,
                                          int32_t element_kind, int64_t rows,
                                          int64_t columns, int64_t nonzeros,
                                          const asc_sb_sparse* destination,
                                          void* workspace,
                                          size_t workspace_bytes);

/* ---- learned variant selector (no reference counterpart) ------------------
 * Twelve features of a matrix (hand-written CUDA kernels) feed a small MLP
 * cost model (12 -> 64 -> 64 -> V, FP32, ReLU) whose output v estimates the
 * log run time of variant v relative to the matrix's mean; the smallest wins.
 * A selector installed on a context picks the variant of every plan created
 * on it in BACKEND_DEFAULT mode with variant AUTO (DETERMINISTIC products
 * always run the bit-exact kernels, so the selector never changes numerics
 * beyond each variant's stated bound).  The training entry points run the
 * MLP's forward pass, backward pass and Adam update on the GPU.
 * Features: log2(1 + rows), log2(1 + columns), log2(1 + nnz),
 * log2(1 + mean row length), log2(1 + max row length), log2(1 + coefficient
 * of variation of row length), max |column - row| / columns, mean |column -
 * row| / columns, diagonal entries / min(rows, columns), nnz / (8 * runs of
 * entries in one 8-column block), empty rows / rows, 1 if double else 0. */
#define ASC_SB_SELECTOR_FEATURES 12
#define ASC_SB_SELECTOR_HIDDEN 64
/* Parameter count for V outputs (1..64), -1 otherwise.  Layout: W1[64][12]
 * b1[64] W2[64][64] b2[64] W3[V][64] b3[V], row-major, FP32. */
ASC_SB_API int64_t asc_sb_selector_param_count(int32_t n_variants);
/* Installs a trained selector (host parameters, copied) whose output i
 * stands for variant variants[i] with lanes[i]; params = NULL removes it. */
ASC_SB_API int asc_sb_context_set_selector(asc_sb_context* context,
                                           int32_t n_variants,
                                           const float* params,
                                           const int32_t* variants,
                                           const int32_t* lanes);
/* Variant recorded in a plan (selector or autotune); AUTO if none. */
ASC_SB_API int asc_sb_plan_variant(const asc_sb_plan* plan, int32_t* variant,
                                   int32_t* lanes);
/* Exhaustive autotune, the selector's fallback and its yardstick: times y = A x with
 * each candidate (one warm-up, `reps` timed runs, CUDA events on the context
 * stream), writes the mean times to ms[count] (nullable) and records the
 * fastest in the plan.  y is overwritten. */
ASC_SB_API int asc_sb_plan_autotune(asc_sb_context* context, asc_sb_plan* plan,
                                    const asc_sb_vector* input,
                                    const asc_sb_vector* output, int32_t count,
                                    const int32_t* variants,
                                    const int32_t* lanes, int32_t reps,
                                    float* ms);
/* The twelve features of a device matrix into `features` (12 device floats);
 * `scratch` is 64 bytes of device memory, 8-byte aligned. */
ASC_SB_API int asc_sb_matrix_features(asc_sb_context* context,
                                      const asc_sb_sparse* matrix,
                                      float* features, void* scratch);
/* Training kernels (device pointers): forward keeps both hidden layers in
 * hidden[batch][128]; backward writes the MSE gradient of every parameter
 * to grads, per-sample losses to loss (nullable), using
 * scratch[batch][V + 128]; Adam updates params, m and v in place. */
ASC_SB_API int asc_sb_selector_forward(asc_sb_context* context,
                                       int32_t n_variants, const float* params,
                                       const float* x, int64_t batch,
                                       float* hidden, float* y);
ASC_SB_API int asc_sb_selector_backward(asc_sb_context* context,
                                        int32_t n_variants,
                                        const float* params, const float* x,
                                        int64_t batch, const float* hidden,
                                        const float* y, const float* target,
                                        float* grads, float* loss,
                                        float* scratch);
ASC_SB_API int asc_sb_selector_adam(asc_sb_context* context, float* params,
                                    const float* grads, float* m, float* v,
                                    int64_t n, float lr, float beta1,
                                    float beta2, float eps, int32_t step);

/* ---- batched SpMV (no reference counterpart) ------------------------------
 * A batch binds `count` independent compat products y_i = alpha A_i x_i +
 * beta y_i (CSR, one element kind: float or double), validated like
 * asc_sb_csr_spmv when the batch is created.  asc_sb_batch_spmv runs all of
 * them as ONE launch of a persistent work-queue kernel: warps take row tiles
 * of any matrix from a global counter, so thousands of uneven matrices share
 * the GPU without a launch per matrix.  DETERMINISTIC contexts get the
 * reference's per-row order and rounding, exactly as asc_sb_csr_spmv.  The
 * batch keeps pointers to the operands: they must stay valid, and no output
 * may overlap another output or any input of the batch.  The workspace
 * (device memory, 256-byte aligned, of the queried size) holds the operand
 * table, the tile bounds and the queue counter for the life of the batch. */
typedef struct asc_sb_batch asc_sb_batch;
ASC_SB_API int asc_sb_batch_workspace_size(asc_sb_context* context,
                                           int64_t count,
                                           const asc_sb_sparse* matrices,
                                           size_t* bytes);
ASC_SB_API int asc_sb_batch_create(asc_sb_context* context, int64_t count,
                                   const asc_sb_sparse* matrices,
                                   const asc_sb_vector* inputs,
                                   const asc_sb_vector* outputs,
                                   void* workspace, size_t workspace_bytes,
                                   asc_sb_batch** out);
ASC_SB_API int asc_sb_batch_destroy(asc_sb_batch* batch);
/* Schedule of the persistent launch: tiles a warp takes per queue grab
 * (1..4096) and CTAs per SM (0 = the occupancy limit, else 1..32). */
ASC_SB_API int asc_sb_batch_set_schedule(asc_sb_context* context,
                                         asc_sb_batch* batch,
                                         int32_t chunk_tiles,
                                         int32_t ctas_per_sm);
ASC_SB_API int asc_sb_batch_get_schedule(const asc_sb_batch* batch,
                                         int32_t* chunk_tiles,
                                         int32_t* ctas_per_sm);
/* All products of the batch in one launch (a replay of the captured graph
 * when asc_sb_batch_capture recorded one for the same alpha, beta,
 * determinism and schedule). */
ASC_SB_API int asc_sb_batch_spmv(asc_sb_context* context, asc_sb_batch* batch,
                                 double alpha, double beta);
/* The same products as one plain-kernel launch per matrix (the baseline). */
ASC_SB_API int asc_sb_batch_spmv_per_matrix(asc_sb_context* context,
                                            asc_sb_batch* batch, double alpha,
                                            double beta);
/* Records the persistent launch (queue reset + kernel) for these scalars
 * into a CUDA graph owned by the batch. */
ASC_SB_API int asc_sb_batch_capture(asc_sb_context* context,
                                    asc_sb_batch* batch, double alpha,
                                    double beta);
/* Times every schedule of the tuning space (`reps` products each, CUDA events
 * on the context stream), keeps the fastest and returns its time per product.
 * The products run for real: outputs are written every time, so with
 * beta != 0 they accumulate. */
ASC_SB_API int asc_sb_batch_autotune(asc_sb_context* context,
                                     asc_sb_batch* batch, double alpha,
                                     double beta, int32_t reps,
                                     float* best_ms);

/* ---- storage sizes for clones into caller-owned memory --------------------- */

/* Byte sizes of the three arrays of a CSR/CSC descriptor after the reference's
 * metadata validation (ValidateSparseMetadata, operations.cc:134-251), so that
 * a binding can allocate a clone's destination from the caller's memory
 * resource -- as CloneCsrErased does (operations.cc:696-731) -- before
 * asc_sb_clone_csr.  Nothing is touched on the device. */
ASC_SB_API int asc_sb_sparse_storage_bytes(asc_sb_context* context,
                                           const asc_sb_sparse* source,
                                           size_t* offsets, size_t* indices,
                                           size_t* values);
/* The same for an indexed vector (ValidateIndexedMetadata,
 * operations.cc:542-570), ahead of asc_sb_clone_indexed
 * (CloneIndexedErased, operations.cc:802-830). */
ASC_SB_API int asc_sb_indexed_storage_bytes(asc_sb_context* context,
                                            const asc_sb_indexed_vector* source,
                                            size_t* indices, size_t* values);

/* ---- pointwise evaluation over one sparsity structure --------------------- */

/* internal_sparse_cuda::PointwiseOperation and OperandKind (cuda.h:130-141). */
enum {
  ASC_SB_POINTWISE_COPY = 0,
  ASC_SB_POINTWISE_NEGATE = 1,
  ASC_SB_POINTWISE_ADD = 2,
  ASC_SB_POINTWISE_SUBTRACT = 3,
  ASC_SB_POINTWISE_MULTIPLY = 4
};
enum { ASC_SB_OPERAND_VIEW = 0, ASC_SB_OPERAND_SCALAR = 1 };

/* internal_sparse_cuda::SparseDescriptor in full (cuda.h:143-156): any rank,
 * for coordinate (ASC_SB_COORDINATE: structure_first holds nonzeros x rank
 * int64 coordinates), CSR and CSC (rank two) storage. */
typedef struct asc_sb_tensor {
  const void* structure_first;
  const void* structure_second;
  const void* values;
  int32_t memory_space;
  int32_t element_kind;
  int32_t format;
  int32_t canonical_structure_trusted;
  int64_t rank;
  const int64_t* extents;  /* rank entries (host memory) */
  int64_t nonzeros;
} asc_sb_tensor;

/* internal_sparse_cuda::OperandDescriptor (cuda.h:158-162): a view with the
 * destination's structure, or a scalar whose element kind is view.element_kind. */
typedef struct asc_sb_operand {
  int32_t kind;
  int32_t reserved;
  asc_sb_tensor view;
  double scalar;
} asc_sb_operand;

/* Replaces internal_sparse_cuda::EvaluateErased (cuda.h:228-231;
 * operations.cc:1051-1120, kernel kernels.cu:118-158): for every stored
 * position p, destination.values[p] = left[p] (copy), -left[p] (negate), or
 * left[p] op right[p] (add, subtract, multiply), where a view operand reads
 * its values at p and a scalar operand is its value converted to the element
 * type.  View operands must share the destination's structure arrays (same
 * pointers, format, rank, extents, nonzeros); a view's values may be the
 * destination's values but may not partially overlap them.  float and
 * double only, as the reference's public template allows. */
ASC_SB_API int asc_sb_evaluate(asc_sb_context* context, int32_t operation,
                               const asc_sb_operand* left,
                               const asc_sb_operand* right,
                               const asc_sb_tensor* destination);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* ASC_SPARSE_B200_H_ */
