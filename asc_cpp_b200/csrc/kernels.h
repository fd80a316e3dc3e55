// Internal launch layer: plain extern "C" entry points from the C++20 host
// code into the sm_100a kernels.  Not part of the public ABI
// (include/asc_sparse_b200.h is).  Every function enqueues on `stream` and
// returns the cudaError_t of the launch (0 on success).
#pragma once

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ascb_csr {
  int64_t rows;
  int64_t cols;
  int64_t nnz;
  const int64_t* ptr;
  const int64_t* idx;
  const void* val;
} ascb_csr;

typedef struct ascb_vec {
  void* data;      // logical element 0
  int64_t n;
  int64_t stride;  // may be negative
} ascb_vec;

// complex kinds hold (re, im) pairs, the layout of std::complex
enum { ASCB_F32 = 0, ASCB_F64 = 1, ASCB_C64 = 2, ASCB_C128 = 3 };
enum { ASCB_COL_MAJOR = 0, ASCB_ROW_MAJOR = 1 };
// Arithmetic forms: COMPAT is y = alpha*(sum v x) + beta*y (reference_blas.cc);
// STANDARD is y += (alpha*v)*x per entry (blas.h:1653-1665).
enum { ASCB_COMPAT = 0, ASCB_STANDARD = 1 };

// ---- partitions (integer work, bit-exact) ----
// Row tiles: tile k owns rows r with weight*r + ptr[r] in
// [k*items, (k+1)*items).  Writes ntiles+1 row bounds.
int64_t ascb_row_tile_count(int64_t rows, int64_t nnz, int64_t items, int64_t weight);
int ascb_row_tiles(void* stream, const ascb_csr* a, int64_t items, int64_t weight,
                   int64_t* tile_row, int64_t ntiles);
// Merge-path split points of diagonals k*items, k = 0..ntiles (row, nnz).
int64_t ascb_merge_tile_count(int64_t rows, int64_t nnz, int64_t items);
int ascb_merge_path_splits(void* stream, const ascb_csr* a, int64_t items,
                           int64_t* split_row, int64_t* split_nz,
                           int64_t ntiles);

// ---- stable sort by key (format conversions, transposed structure) ----
// perm[q] = source position of the q-th entry in (key, position) order of
// keys[e * kstride], e < n; offsets[0..limit] = bucket starts (keys outside
// [0, limit) are not counted).  `workspace` holds ascb_sort_workspace_bytes.
size_t ascb_sort_workspace_bytes(int64_t n, int64_t limit);
int ascb_stable_sort(void* stream, const int64_t* keys, int64_t kstride, int64_t n, int64_t limit,
                     int64_t* offsets, int64_t* perm, void* workspace);
// out[q] = r for every entry q in [ptr[r], ptr[r+1]).
int ascb_outer_of_entries(void* stream, const int64_t* ptr, int64_t outer, int64_t* out,
                          int sm_count);
// idx_out[j] = other[perm[j] * ostride] (if idx_out), val_out[j] =
// val_in[perm[j]] (if val_out; elem_bytes 4, 8 or 16).
int ascb_permute_entries(void* stream, const int64_t* perm, int64_t n, const int64_t* other,
                         int64_t ostride, int64_t* idx_out, const void* val_in, void* val_out,
                         int elem_bytes, int sm_count);

// ---- SpMV variants ----
// Warp-tiled SpMV over row tiles of ascb_warp_tile_items() weighted items with
// row weight ascb_warp_tile_row_weight().  exact = 1 reproduces the serial
// reference bit for bit.  tile_row may be NULL (bounds searched in-kernel).
int64_t ascb_warp_tile_items(void);
int64_t ascb_warp_tile_row_weight(void);
int ascb_spmv_warp(void* stream, int dtype, int form, int exact, const ascb_csr* a,
                   double alpha, double beta, const ascb_vec* x, const ascb_vec* y,
                   const int64_t* tile_row, int64_t ntiles, int sm_count);
// Register-segmented SpMV over the warp row tiles (exact = 1: bit-exact);
// requires the column-index and value arrays to start on
// ascb_spmv_seg_alignment()-byte boundaries.
int ascb_spmv_seg_alignment(void);
int ascb_spmv_seg(void* stream, int dtype, int form, int exact, const ascb_csr* a, double alpha,
                  double beta, const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
                  int64_t ntiles, int sm_count);
// The same over row tiles of weight `weight`: ascb_warp_tile_row_weight() (at
// most 32 rows per tile, as ascb_spmv_seg) or ascb_seg_tile_row_weight() (the
// segmented kernel's own partition: more rows per tile, so more of each
// window holds nonzeros when rows are short).
int64_t ascb_seg_tile_row_weight(void);
// Weighted items per tile of that partition (ascb_row_tiles' `items`): fewer
// than ascb_warp_tile_items() when the weight is small, so that every row of
// a tile but the first starts inside the tile's 256-position window.
int64_t ascb_seg_tile_items(void);
// The merge partition for the segmented kernel (MERGE_PATH): weight 1 (one
// item per row and one per nonzero), at most ascb_merge_tile_items() items a
// tile; ascb_spmv_seg_w runs it with exact = 0 only.
int64_t ascb_merge_tile_row_weight(void);
int64_t ascb_merge_tile_items(void);
int ascb_spmv_seg_w(void* stream, int dtype, int form, int exact, const ascb_csr* a, double alpha,
                    double beta, const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
                    int64_t ntiles, int64_t weight, int sm_count);
// Row split (contracted only): like ascb_spmv_seg with exact = 0, except that
// a row running more than split_min (>= 256) positions past its tile's window
// is finished by a second kernel whose warps take its tail in 256-position
// chunks; partial sums are combined in chunk order, so results repeat run to
// run.  `block`: ascb_split_bytes(nnz, split_min) device bytes, 256-byte
// aligned (its control words are cleared on the stream by the call).
size_t ascb_split_bytes(int64_t nnz, int64_t split_min);
int ascb_spmv_split(void* stream, int dtype, int form, const ascb_csr* a, double alpha,
                    double beta, const ascb_vec* x, const ascb_vec* y, const int64_t* tile_row,
                    int64_t ntiles, int64_t weight, int64_t split_min, void* block,
                    int sm_count);
// ---- batched compat SpMV: many independent CSR matrices, one launch ----
// One matrix of a batch, as the persistent kernel reads it (device table).
typedef struct ascb_batch_item {
  const int64_t* ptr;
  const int64_t* idx;
  const void* val;
  const void* x;        // logical element 0
  void* y;              // logical element 0
  int64_t rows;
  int64_t nnz;
  int64_t incx;
  int64_t incy;
  int64_t tile_base;    // first global tile of this matrix
  int64_t bound_base;   // first entry of its tile bounds (tile_base + index)
} ascb_batch_item;
// Tile bounds of every matrix: bounds[bound_base + k] = first row of tile k,
// k = 0..tiles (the last entry is rows).  `items` is the device table.
int ascb_batch_tile_bounds(void* stream, const ascb_batch_item* items, int64_t count,
                           int64_t* bounds, int64_t total_bounds, int sm_count);
// Persistent work-queue SpMV over all tiles of the batch: warps take `chunk`
// tiles at a time from *queue (zero before the launch); ctas_per_sm = 0 uses
// the occupancy limit.  Index and value arrays must be 16-byte aligned.
int ascb_spmv_seg_batch(void* stream, int dtype, int exact, int unit,
                        const ascb_batch_item* items, int64_t count, const int64_t* bounds,
                        int64_t total_tiles, unsigned long long* queue, int chunk,
                        int ctas_per_sm, double alpha, double beta, int sm_count);

// ---- learned variant selector (features + MLP cost model) ----
#define ASCB_SELECTOR_FEATURES 12
#define ASCB_SELECTOR_HIDDEN 64
int64_t ascb_mlp_param_count(int n_variants);
// acc: 8 device uint64 of scratch; features: 12 device floats.
int ascb_matrix_features(void* stream, const ascb_csr* a, int element_bytes,
                         unsigned long long* acc, float* features, int sm_count);
// hidden: batch * 128 floats (both hidden layers, kept for the backward pass).
int ascb_mlp_forward(void* stream, int n_variants, const float* params, const float* x,
                     int64_t batch, float* hidden, float* y);
// grads: ascb_mlp_param_count floats; loss (nullable): batch floats;
// scratch: batch * (n_variants + 128) floats.
int ascb_mlp_backward(void* stream, int n_variants, const float* params, const float* x,
                      int64_t batch, const float* hidden, const float* y, const float* target,
                      float* grads, float* loss, float* scratch);
int ascb_adam_step(void* stream, float* params, const float* grads, float* m, float* v,
                   int64_t n, float lr, float beta1, float beta2, float eps, int step);
int ascb_argmin(void* stream, const float* y, int n, int* out);

// Vector CSR: `lanes` (1..32, power of two) threads per row.
int ascb_spmv_vector(void* stream, int dtype, int form, int lanes,
                     const ascb_csr* a, double alpha, double beta,
                     const ascb_vec* x, const ascb_vec* y, int sm_count);

// Transposed SpMV by scatter: y[c] += alpha * v * x[r] with atomics.
int ascb_spmv_scatter(void* stream, int dtype, const ascb_csr* a, double alpha,
                      const ascb_vec* x, const ascb_vec* y, int sm_count);

// ---- complex standard products (dtype ASCB_C64 / ASCB_C128) ----
// mode 0: rows of `a`, any summation order; 1: rows of `a`, the reference's
// order and rounding; 2: scatter of the transpose of `a` (atomics).  conj = 1
// conjugates the stored values.
int ascb_complex_spmv(void* stream, int dtype, int mode, int conj, const ascb_csr* a,
                      double alpha_re, double alpha_im, const ascb_vec* x, const ascb_vec* y,
                      int sm_count);
int ascb_complex_spmm(void* stream, int dtype, int mode, int conj, const ascb_csr* a, int64_t k,
                      const void* b, int b_layout, int64_t ldb, void* c, int c_layout,
                      int64_t ldc, double alpha_re, double alpha_im, int sm_count);

// ---- block-sparse SpMM on tensor cores (16 x 16 dense blocks, FP32) ----
// *bad (device int) becomes 1 unless every block row of `a` (rows a multiple
// of 16) is made of dense, aligned 16 x 16 blocks.
int ascb_block16_check(void* stream, const ascb_csr* a, int* bad, int sm_count);
size_t ascb_block16_tc_smem(void);
// C += alpha * A * B, row-major B (ldb) and C (ldc); values 16-byte aligned;
// 3xTF32 on tcgen05.  `tiles`: ascb_block16_tiles_bytes(a->cols, k) device
// bytes, 256-byte aligned, for the B^T tile images the call's pre-pass
// writes.  status (nullable) receives 1 if a bounded wait gave up.
size_t ascb_block16_tiles_bytes(int64_t cols, int64_t k);
int ascb_spmm_block16_tc(void* stream, const ascb_csr* a, int64_t k, const float* b,
                         int64_t ldb, float* c, int64_t ldc, float alpha, float* tiles,
                         int* status, int sm_count);

// ---- Level-1 on an indexed vector (internal_sparse_cuda::StandardOperation) ----
enum { ASCB_L1_DOT = 0, ASCB_L1_AXPY = 1, ASCB_L1_GATHER = 2, ASCB_L1_GATHER_ZERO = 3,
       ASCB_L1_SCATTER = 4 };
#define ASCB_L1_DOT_BLOCKS 256
// idx/val: n entries; x: dense vector (logical element 0, stride incx);
// result: one element (dot).  exact = 1: the reference's order and rounding
// for the dot.  scratch: ASCB_L1_DOT_BLOCKS elements for the contracted dot.
int ascb_level1(void* stream, int dtype, int op, int conj, int exact, const int64_t* idx,
                void* val, int64_t n, void* x, int64_t incx, void* result, double alpha_re,
                double alpha_im, void* scratch, int sm_count);

// ---- sparse triangular solve op(A) X = alpha B, X over B ----
// ptr/idx/val: CSR of M = op(A) (n x n, sorted columns; values already those
// of op(A) up to conjugation, applied when conj = 1).  lower: M is lower
// triangular (rows solved 0..n-1), else upper (n-1..0); order/position
// (nullable, from ascb_trsv_analysis) replace that order by a level order.
// x: the n x k dense right-hand sides, element (r, j) at r*ld + j (row_major)
// or j*ld + r.  control: ascb_trsv_scratch_bytes(n, element bytes) device
// bytes, 16-byte aligned, prepared by the call on the stream; pub = control +
// 16 bytes.  status (nullable) receives 1 if a bounded wait gave up.
typedef struct ascb_trsv {
  const int64_t* ptr;
  const int64_t* idx;
  const void* val;
  int64_t n;
  int lower, unit, conj, row_major;
  void* x;
  int64_t ld;
  int64_t k;
  void* control;
  void* pub;
  const int64_t* order;
  const int64_t* position;
  int* status;
  uint64_t wait_ns;  // longest wait on one dependency; 0: 2 s
} ascb_trsv;
size_t ascb_trsv_scratch_bytes(int64_t n, int elem_bytes);
// exact = 1: the reference's order and rounding (DETERMINISTIC).
// alpha_is_zero = 1: X = 0 without reading it.
int ascb_sptrsv(void* stream, int dtype, int exact, int alpha_is_zero, const ascb_trsv* t,
                double alpha_re, double alpha_im, int sm_count);
// Level order of M (t: ptr, idx, n, lower, control, status): rows sorted by
// dependency level, stable by row.  workspace: ascb_trsv_analysis_bytes(n),
// 256-byte aligned; *order / *position point into it (solve position -> row
// and row -> solve position).
size_t ascb_trsv_analysis_bytes(int64_t n);
int ascb_trsv_analysis(void* stream, const ascb_trsv* t, void* workspace, int64_t** order,
                       int64_t** position, int sm_count);

// ---- SpMM: C += alpha * op(A) * B (k right-hand sides) ----
// transpose = 0: stored-order row kernels (exact = 1: the reference's order
// and rounding; 0: contracted); 1: atomic scatter.
int ascb_spmm(void* stream, int dtype, int transpose, int exact, const ascb_csr* a,
              int64_t k, const void* b, int b_layout, int64_t ldb, void* c,
              int c_layout, int64_t ldc, double alpha, int sm_count);

// ---- row-group SpMM (plan-built runs of R consecutive rows) ----
// A plan's row groups: runs (distinct columns of each group of R rows, in
// column order) with the rows that hold them and their values.
typedef struct ascb_row_groups {
  int rows_per_group;         // R: 2, 4, 8, 16 or 32
  int64_t* group_runs;        // [groups + 1]
  int64_t* run_col;           // [runs]
  unsigned* run_mask;         // [runs] bit i: row g*R + i holds the column
  unsigned* run_off;          // [runs] first value, relative to ptr[g*R]
  void* vals;                 // [nnz] values in (group, column, row) order
} ascb_row_groups;
typedef struct ascb_row_groups_layout {
  size_t group_runs, run_col, run_mask, run_off, vals, persistent;
  size_t row_of, perm, flags, run_of, sums, total;
} ascb_row_groups_layout;
// Byte offsets in a 256-byte aligned block serving any R (at most
// rows/2 + 1 groups, at most nnz runs); [persistent, total) is build scratch.
ascb_row_groups_layout ascb_row_groups_layout_for(int64_t rows, int64_t nnz, int elem_bytes);
// Builds the groups of CSR `a` (sorted columns) for R rows per group in
// `base`; enqueued on the stream (integer work, deterministic).
int ascb_row_groups_build(void* stream, const ascb_csr* a, int elem_bytes, int rows_per_group,
                          void* base, ascb_row_groups* out, int sm_count);
// C += alpha * A * B, row-major B and C with 16-byte aligned rows (k, ldb and
// ldc multiples of 16 bytes / element); exact = 1: the reference's per-entry
// update in stored order (bit-exact).
int ascb_spmm_groups(void* stream, int dtype, int exact, const ascb_csr* a,
                     const ascb_row_groups* rg, int64_t k, const void* b, int64_t ldb, void* c,
                     int64_t ldc, double alpha, int sm_count);

// Exclusive scan of n int64 values: out[i] = in[0] + ... + in[i-1] for
// i <= n (out holds n + 1); `sums`: (n / 2048 + 2) int64 of scratch.
int ascb_scan_i64(void* stream, const int64_t* in, int64_t n, int64_t* out, int64_t* sums);

// ---- TMA-staged SpMM (plan-built groups of 16, 32 and 64 rows) ----
// Per group of rows: its distinct columns ("slots", column order), their
// maximal runs of consecutive columns ("segments"), and per stored entry the
// slot of its column.  Three levels: groups of 16 rows, and wide groups of 32
// and 64 (two or four groups merged: a column they share is one slot).
#define ASCB_STAGED_LEVELS 3
typedef struct ascb_staged_spmm {
  int64_t groups;
  int64_t group_rows;   // 16, 32 or 64
  int64_t* group_runs;  // [groups + 1] slots before each group
  int64_t* group_segs;  // [groups + 1] segments before each group
  int64_t* seg_col;     // [segments] first column
  int64_t* seg_run;     // [segments] first slot, numbered over all groups
  int32_t* seg_len;     // [segments] columns
  uint16_t* slot;       // [nnz] group-relative slot of each entry's column
  // device words: largest slot and entry counts over aligned windows of
  // 1, 2, 4, 8, 16 groups (pairs, in that order)
  unsigned long long* caps;
} ascb_staged_spmm;
typedef struct ascb_staged_level_layout {
  size_t group_runs, group_segs, seg_col, seg_run, seg_len, slot, caps;
} ascb_staged_level_layout;
typedef struct ascb_staged_layout {
  ascb_staged_level_layout level[ASCB_STAGED_LEVELS];  // 16, 32, 64 rows
  size_t persistent;
  size_t seg_flag, seg_of, sums, wide_slot_of, wide_col, total;
} ascb_staged_layout;
// Byte offsets in a 256-byte aligned block; [persistent, total) is build
// scratch.
ascb_staged_layout ascb_staged_layout_for(int64_t rows, int64_t nnz);
// Builds every level's tables (levels[0 .. ASCB_STAGED_LEVELS): groups of
// 16, 32, 64 rows) from row groups of 16 rows just built by
// ascb_row_groups_build into `groups_base` (it reads that build's scratch).
int ascb_staged_build(void* stream, const ascb_csr* a, const ascb_row_groups* rg16,
                      const void* groups_base, int elem_bytes, void* base,
                      ascb_staged_spmm* levels, int sm_count);
// Groups per pipeline stage for k right-hand sides (a stage holds at least
// the rows one pass of the consumers covers), and the bytes of one stage
// holding `slots` rows of B and `entries` stored entries.
int ascb_staged_groups_per_stage(int dtype, int64_t k, int64_t group_rows);
size_t ascb_staged_stage_bytes(int dtype, int64_t k, int64_t slots, int64_t entries, int ng,
                               int64_t group_rows);
// C += alpha * A * B (row-major B and C, rows of whole 16-byte chunks on
// 16-byte boundaries) over the groups of `st` (either level); max_slots /
// max_entries: the caps of the stage width ascb_staged_groups_per_stage;
// exact = 1: the reference's per-entry update in stored order (bit-exact).
// Two stages of ascb_staged_stage_bytes each must fit one CTA's shared memory.
int ascb_spmm_staged(void* stream, int dtype, int exact, const ascb_csr* a,
                     const ascb_staged_spmm* st, int64_t k, const void* b, int64_t ldb, void* c,
                     int64_t ldc, double alpha, int64_t max_slots, int64_t max_entries,
                     int* status, int sm_count);

#ifdef __cplusplus
}
#endif
