// Internal interface between the plan (plan.cu) and the kernel files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace rvsp {

// Row classes.  A row is classed twice: for the symbolic pass by the upper
// bound ub = min(ops_i, b_cols) on its output nnz, and for the numeric pass
// by its exact output nnz m_i.  The same table serves both.
//
//   EMPTY   no products
//   M<K>    at most K (4, 8, 16, 32) A nonzeros and at most kMergeMaxOps
//           products: one thread merges the row's K sorted B rows, taking
//           the smallest head column each step; equal heads are added in
//           A-nonzero order, and columns come out sorted with no scratch
//   W<T>    one warp, shared-memory hash table of T slots (bound <= T/2)
//   B8192   one 256-thread block, hash table of 8192 slots (bound <= 4096)
//   DENSE   one 512-thread block, dense accumulator over all of B's columns
enum RowClass : int {
  kEmpty_ = 0,
  kM4,
  kM8,
  kM16,
  kM32,
  kW64,
  kW128,
  kW256,
  kW512,
  kW1024,
  kW2048,
  kB8192,
  kDense,
  kNumClasses
};

constexpr int kMergeMaxOps = 2048;
constexpr int kMergeThreads = 128;
constexpr int kWarpHashMinLog2 = 6;    // W64
constexpr int kWarpHashMaxLog2 = 11;   // W2048
constexpr int kBlockHashLog2 = 13;     // B8192
constexpr int kBlockHashThreads = 256;
constexpr int kDenseThreads = 512;
constexpr int kWarpsPerBlock = 4;      // warp-per-row kernels
// Dense rows keep their column bitmap in shared memory up to this many
// columns (48 Ki words = 192 KiB), else in global scratch.
constexpr int64_t kSmemBitmapMaxCols = 48 * 1024 * 32;
// rowstats hands rows with more A nonzeros than this to a warp-per-row pass.
constexpr int kLongRowNnz = 128;

__host__ __device__ inline int classify_row(int32_t nnz_a, int64_t ops,
                                            int64_t bound) {
  if (ops <= 0) return kEmpty_;
  if (nnz_a <= 32 && ops <= kMergeMaxOps)
    return nnz_a <= 4 ? kM4 : nnz_a <= 8 ? kM8 : nnz_a <= 16 ? kM16 : kM32;
  const int64_t need = 2 * bound;
  for (int l = kWarpHashMinLog2; l <= kWarpHashMaxLog2; ++l)
    if (need <= (int64_t(1) << l)) return kW64 + (l - kWarpHashMinLog2);
  if (bound <= (int64_t(1) << (kBlockHashLog2 - 1))) return kB8192;
  return kDense;
}

inline int class_log2(int cls) { return kWarpHashMinLog2 + (cls - kW64); }

// Pointers of one product.  A's columns index B's rows.
struct Operands {
  int32_t a_rows;
  int32_t b_cols;
  const int32_t *a_rp;
  const int32_t *a_col;
  const float *a_val;
  const int32_t *b_rp;
  const int32_t *b_col;
  const float *b_val;
};

// ---- k_rowstats.cu ---------------------------------------------------------
// ops[i] = sum of B row lengths over A row i; cls[i] = symbolic class of the
// row; class_count[c] += rows per class; counts[i] = 0 for empty rows.
void launch_rowstats(const Operands &op, int64_t *ops, uint8_t *cls,
                     int32_t *counts, int32_t *class_count, int32_t *long_rows,
                     int32_t *long_count, int32_t max_long, cudaStream_t s);
void launch_rowstats_long(const Operands &op, const int32_t *long_rows,
                          const int32_t *long_count, int64_t *ops, uint8_t *cls,
                          int32_t *counts, int32_t *class_count, int num_sms,
                          cudaStream_t s);
// off[c] = exclusive prefix of count over the non-empty classes.
void launch_class_offsets(const int32_t *count, int32_t *off, cudaStream_t s);
// rows_by_class[class_off[c] + r] = i for every non-empty row i of class c.
void launch_scatter_rows(int32_t n, const uint8_t *cls, const int32_t *class_off,
                         int32_t *class_fill, int32_t *rows_by_class,
                         cudaStream_t s);

// ---- k_scan.cu -------------------------------------------------------------
// row_ptr = exclusive scan of counts (n + 1 entries), *total = sum (int64).
// Also classes every row for the numeric pass (cls, class_count).
size_t scan_partials_bytes(int32_t n);
void launch_scan_and_class(int32_t n, const int32_t *counts, const int64_t *ops,
                           const int32_t *a_rp, int32_t *row_ptr,
                           int64_t *partials, int64_t *total, uint8_t *cls,
                           int32_t *class_count, cudaStream_t s);

// ---- k_merge.cu ------------------------------------------------------------
// Thread-per-row K-way merge for the M<K> classes: counts (symbolic) or
// values and sorted columns (numeric).
void launch_merge_symbolic(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, cudaStream_t s);
void launch_merge_numeric(int cls, const Operands &op, const int32_t *rows,
                          int32_t nrows, const int32_t *c_rp, int32_t *c_col,
                          float *c_val, bool fill, int32_t *status,
                          cudaStream_t s);

// ---- k_symbolic.cu ---------------------------------------------------------
// counts[row] = nnz of output row, for the rows of one class.
void launch_symbolic_class(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, uint32_t *gbitmap,
                           int32_t gbitmap_slots, int32_t *status, int num_sms,
                           cudaStream_t s);

// ---- k_check.cu ------------------------------------------------------------
// *result (initialised to ~0ull) receives min over bad rows of
// ((row + 1) << 8 | code); row -1 means row_ptr[0] != 0.
void launch_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                      const int32_t *col_idx, int32_t nnz,
                      unsigned long long *result, cudaStream_t s);

// ---- k_numeric.cu ----------------------------------------------------------
// Values (and, when fill, sorted columns) of the rows of one class.
void launch_numeric_class(int cls, const Operands &op, const int64_t *ops,
                          const int32_t *rows, int32_t nrows,
                          const int32_t *c_rp, int32_t *c_col, float *c_val,
                          bool fill, float *dense_acc, uint32_t *dense_bits,
                          int32_t dense_slots, int32_t *status, int num_sms,
                          cudaStream_t s);
// Global scratch one dense numeric slot needs (accumulator + bitmap if the
// bitmap does not fit shared memory), 256-byte aligned.
size_t dense_slot_acc_bytes(int32_t b_cols);
size_t dense_slot_bits_bytes(int32_t b_cols);

}  // namespace rvsp
