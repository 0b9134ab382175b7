// Internal interface between the plan (plan.cu) and the kernel files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>
#include <cuda_runtime.h>

struct rvsp_mlp;

namespace rvsp {

// Device pointer of a model's parameters (model.cu).
const float *mlp_device_params(const rvsp_mlp *m);

// Row classes.  A row is classed twice: for the symbolic pass by the upper
// bound ub = min(ops_i, b_cols) on its output nnz, and for the numeric pass
// by its exact output nnz m_i.  The same table serves both.
//
//   EMPTY   no products
//   M<K>    at most K (4, 8, 16) A nonzeros and at most kMergeMaxOps
//           products, in a matrix of at least kMergeMinRows rows: one thread
//           merges the row's K sorted B rows, taking the smallest head
//           column each step; equal heads are added in A-nonzero order, and
//           columns come out sorted with no scratch
//   W<T>    one warp, shared-memory hash table of T slots (bound <= T/2)
//   B8192   one 256-thread block, hash table of 8192 slots (bound <= 4096)
//   DENSE   one 512-thread block, dense accumulator over all of B's columns
enum RowClass : int {
  kEmpty_ = 0,
  kM4,
  kM8,
  kM16,
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
constexpr int kMergeMaxNnz = 16;
constexpr int kMergeThreads = 128;
// The merge classes put one row on one thread; below this many rows the GPU
// would sit mostly idle, so smaller matrices use the warp-per-row classes.
constexpr int32_t kMergeMinRows = 32768;
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

// merge_ok: the matrix has at least kMergeMinRows rows.
__host__ __device__ inline int classify_row(int32_t nnz_a, int64_t ops,
                                            int64_t bound, bool merge_ok) {
  if (ops <= 0) return kEmpty_;
  if (merge_ok && nnz_a <= kMergeMaxNnz && ops <= kMergeMaxOps)
    return nnz_a <= 4 ? kM4 : nnz_a <= 8 ? kM8 : kM16;
  const int64_t need = 2 * bound;
  for (int l = kWarpHashMinLog2; l <= kWarpHashMaxLog2; ++l)
    if (need <= (int64_t(1) << l)) return kW64 + (l - kWarpHashMinLog2);
  if (bound <= (int64_t(1) << (kBlockHashLog2 - 1))) return kB8192;
  return kDense;
}

inline int class_log2(int cls) { return kWarpHashMinLog2 + (cls - kW64); }
inline bool is_merge_class(int cls) { return cls == kM4 || cls == kM8 || cls == kM16; }

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
  // Rows may take the merge classes (set by the plan from its merge policy
  // and the row count; see classify_row).
  bool merge_ok;
  // When >= 0: A's entry count and B's row count, which bound every index
  // the row statistics read, so they run safely on structure whose device
  // check has not finished yet (rvsp_cuda_symbolic_checked).
  int32_t a_nnz = -1;
  int32_t b_rows = -1;
};

// The device-side verdict of CSR checks queued earlier on the same stream:
// n words at w, each ~0ull when its structure passed.  A pass given a guard
// that failed returns without reading the structure or writing anything, so
// it can be queued before the verdict reaches the host.  n == 0: no check.
struct CheckGuard {
  const unsigned long long *w = nullptr;
  int n = 0;
#ifdef __CUDACC__
  __device__ __forceinline__ bool failed() const {
    for (int i = 0; i < n; ++i)
      if (w[i] != ~0ull) return true;
    return false;
  }
#endif
};

// Merge policies of a plan: automatic (merge classes when the matrix has at
// least kMergeMinRows rows), never, or whenever a row is eligible.
enum MergePolicy : int { kMergeAuto = 0, kMergeNever = 1, kMergeAlways = 2 };

inline bool merge_allowed(int policy, int32_t a_rows) {
  return policy == kMergeAlways || (policy == kMergeAuto && a_rows >= kMergeMinRows);
}

// Where the fused (learned) pass writes each row: a slot of fo.cap[row]
// entries at fo.off[row] in the slab (the c_col / c_val pointers of the fill
// kernels).  The kernel writes the row's nnz to fo.counts[row], or -1 and
// appends the row to ovf_rows when it needs more than its capacity.
struct FusedOut {
  const int64_t *off;
  const int32_t *cap;
  int32_t *counts;
  int32_t *ovf_rows;
  int32_t *ovf_count;
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
// Also classes every row for the numeric pass (cls, class_count); rows with
// skip[row] >= 0 (the shift-class members) are classed empty.  With a guard
// that failed, nothing is written but the tile partials.
size_t scan_partials_bytes(int32_t n);
void launch_scan_and_class(int32_t n, const int32_t *counts, const int64_t *ops,
                           const int32_t *a_rp, int32_t *row_ptr,
                           int64_t *partials, int64_t *total, uint8_t *cls,
                           int32_t *class_count, bool merge_ok, cudaStream_t s,
                           CheckGuard guard = CheckGuard(), const int32_t *skip = nullptr);

// out[i] = sum of in[0..i) as int64 (n entries), *total = sum of all.
void launch_scan_i64(int32_t n, const int32_t *in, int64_t *out, int64_t *partials,
                     int64_t *total, cudaStream_t s);

// ---- k_fused.cu ------------------------------------------------------------
// Copies every non-overflowed row (counts[row] >= 0) from its slab slot to C
// at row_ptr[row]; values too when with_values.  big: scratch of a_rows + 1
// words (count and list of the rows copied by whole blocks).
void launch_compact(int32_t a_rows, const int32_t *counts, const int64_t *off,
                    const int32_t *row_ptr, const int32_t *slab_col,
                    const float *slab_val, int32_t *c_col, float *c_val,
                    bool with_values, int32_t *big, int num_sms, cudaStream_t s);
// Classes the rows of a list (symbolic: by ub = min(ops, b_cols); numeric: by
// exact nnz counts[row]); cls_out[j] for list entry j; class_count += rows.
void launch_list_classify(const int32_t *list, int32_t n, const int64_t *ops,
                          const int32_t *a_rp, const int32_t *counts, int32_t b_cols,
                          bool numeric, uint8_t *cls_out, int32_t *class_count,
                          cudaStream_t s);
// out[off[c] + r] = list[j] for the entries j of class c (any order).
void launch_scatter_list(const int32_t *list, int32_t n, const uint8_t *cls,
                         const int32_t *class_off, int32_t *class_fill, int32_t *out,
                         cudaStream_t s);
// Order-independent 64-bit fingerprint of n floats added into *h.
void launch_values_hash(const float *v, int64_t n, unsigned long long salt,
                        unsigned long long *h, cudaStream_t s);

// ---- k_merge.cu ------------------------------------------------------------
// Thread-per-row K-way merge for the M<K> classes: counts (symbolic) or
// values and sorted columns (numeric).
void launch_merge_symbolic(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, cudaStream_t s);
// The symbolic pass of every M4, M8 and M16 row, with no row lists and no
// host-side class counts: one launch per merge class over all a_rows rows,
// each thread skipping rows whose cls is another class.  Three launches.
void launch_merge_symbolic_all(const Operands &op, const uint8_t *cls, int32_t a_rows,
                               int32_t *counts, CheckGuard guard, cudaStream_t s);
void launch_merge_numeric(int cls, const Operands &op, const int32_t *rows,
                          int32_t nrows, const int32_t *c_rp, int32_t *c_col,
                          float *c_val, bool fill, int32_t *status,
                          const FusedOut *fo, cudaStream_t s);

// ---- k_symbolic.cu ---------------------------------------------------------
// W1024 / W2048 rows: counted first in a 512-slot table with bounded probes;
// rows that do not fit go to retry[] (count at *retry_n, zeroed by the
// caller, room for nrows) and are counted at their class size.
bool symbolic_optimistic_class(int cls);
void launch_symbolic_optimistic(int cls, const Operands &op, const int32_t *rows,
                                int32_t nrows, int32_t *counts, int32_t *retry,
                                int32_t *retry_n, int32_t *status, int num_sms,
                                cudaStream_t s);
// counts[row] = nnz of output row, for the rows of one class.
void launch_symbolic_class(int cls, const Operands &op, const int32_t *rows,
                           int32_t nrows, int32_t *counts, uint32_t *gbitmap,
                           int32_t gbitmap_slots, int32_t *status, int num_sms,
                           cudaStream_t s);

// ---- k_heavy.cu ------------------------------------------------------------
// B8192 and DENSE rows when B has at most kHeavyMaxCols columns: block per
// row, shared-memory column bitmap, accumulation at output positions.
constexpr int32_t kHeavyMaxCols = 1 << 20;
bool heavy_fits(int32_t b_cols);
void launch_heavy_symbolic(const Operands &op, const int32_t *rows, int32_t nrows,
                           int32_t *counts, int num_sms, cudaStream_t s);
// fill: write C's sorted columns too (fo: the fused pass's slab slots, with
// overflow when a row needs more than its capacity); else reuse C's columns.
void launch_heavy_numeric(const Operands &op, const int32_t *rows, int32_t nrows,
                          const int32_t *c_rp, int32_t *c_col, float *c_val, bool fill,
                          int32_t *status, const FusedOut *fo, int num_sms,
                          cudaStream_t s);

// ---- k_reuse.cu ------------------------------------------------------------
// Reuse map of the W<T> classes: per product, its position in C's row.
bool map_class(int cls);
// mops[row] = ops[row] for the listed rows (the caller zeroes mops);
// *too_long |= 1 when a row has more than INT32_MAX / 2 products.
void launch_map_ops(const int32_t *rows, int32_t nrows, const int64_t *ops, int32_t *mops,
                    int32_t *too_long, cudaStream_t s);
// map[moff[row] + t] = position in C's row of the row's t-th product;
// key[row] (when key is not null) = fingerprint of the row's map, 0 when the
// row met a missing column.
void launch_map_build(int cls, const Operands &op, const int32_t *rows, int32_t nrows,
                      const int32_t *c_rp, const int32_t *c_col, const int64_t *moff,
                      uint16_t *map, unsigned long long *key, int32_t *status,
                      cudaStream_t s);
// Sharing of identical maps: insert every listed row's key into the table
// (tkey zeroed, trow filled with 0x7f bytes, mask + 1 a power of two at least
// twice the rows inserted over all calls); then resolve, which points
// moff[row] at the map of the smallest row c with an identical map, sets
// canon[row] = c (row itself when no other row shares its map, -1 for a row
// without a fingerprint), adds 1 to share_count[c] (zeroed by the caller)
// and the rows so redirected to *shared_rows.
void launch_map_dedup_insert(const int32_t *rows, int32_t nrows,
                             const unsigned long long *key, unsigned long long *tkey,
                             int32_t *trow, unsigned long long mask, cudaStream_t s);
void launch_map_dedup_resolve(const int32_t *rows, int32_t nrows,
                              const unsigned long long *key,
                              const unsigned long long *tkey, const int32_t *trow,
                              unsigned long long mask, const int32_t *c_rp,
                              const int32_t *mops, int64_t *moff, const uint16_t *map,
                              int32_t *shared_rows, int32_t *canon, int32_t *share_count,
                              cudaStream_t s);
// Values of the listed rows of class cls from the map (structure in C).
void launch_map_numeric(int cls, const Operands &op, const int64_t *ops, const int32_t *rows,
                        int32_t nrows, const int32_t *c_rp, float *c_val,
                        const int64_t *moff, const uint16_t *map, int32_t *status,
                        cudaStream_t s);

// ---- k_pattern.cu ----------------------------------------------------------
// Term tables of the rows that share a reuse map (see k_pattern.cu).
// Select: canonical rows shared by at least min_share rows (itself included)
// whose row fits a table get pat_of[row] = id (pat_of filled with -1 by the
// caller), pat_canon[id], pat_cap[id] records; *npat counts them;
// maxima[0] / maxima[1] (zeroed by the caller) receive the largest products
// (rounded up to 32) and C row of the tables.
void launch_pat_select(const int32_t *rows, int32_t nrows, const int32_t *canon,
                       const int32_t *share_count, int32_t min_share, const int32_t *a_rp,
                       const int32_t *c_rp, const int32_t *mops, int32_t *pat_of,
                       int32_t *pat_canon, int32_t *pat_cap, int32_t *npat, int32_t *maxima,
                       cudaStream_t s);
// Build: the npat tables at rec + pat_off[id]; psteps[id] = steps, or -1.
void launch_pat_build(int32_t npat, const int32_t *pat_canon, const int32_t *a_rp,
                      const int32_t *a_col, const int32_t *b_rp, const int32_t *c_rp,
                      const int64_t *moff, const uint16_t *map, const int64_t *pat_off,
                      const int32_t *pat_cap, uint32_t *rec, int32_t *psteps,
                      cudaStream_t s);
// Split a class's rows into table rows (pat_rows / pat_ids, appended at
// *pat_n; pid_of_row[row] = id when pid_of_row is not null) and the rest
// (res_rows, appended at *res_n).
void launch_pat_split(const int32_t *rows, int32_t nrows, const int32_t *canon,
                      const int32_t *pat_of, const int32_t *psteps, const int32_t *a_rp,
                      const int32_t *a_col, const int32_t *b_rp, int32_t *pat_rows,
                      int32_t *pat_ids, int32_t *pat_n, int32_t *res_rows, int32_t *res_n,
                      int32_t *pid_of_row, cudaStream_t s);
// Values of the n table rows (structure in C); max_ops / max_out: the
// maxima the select step found.
void launch_pat_numeric(const Operands &op, const int64_t *ops, const int32_t *pat_rows,
                        const int32_t *pat_ids, int32_t n, const int32_t *c_rp, float *c_val,
                        const int64_t *pat_off, const int32_t *psteps, const uint32_t *rec,
                        int32_t max_ops, int32_t max_out, cudaStream_t s);

// ---- k_tile.cu -------------------------------------------------------------
// Row tiles of the table rows (see k_tile.cu).  Warps per block of the tile
// kernel; uint16 entries per pattern in
// the tile tables (tab has npat * tile_tab_stride() entries).
constexpr int kTileKernelWarps = 2;
int32_t tile_tab_stride();
// Per pattern: its table, B row lengths (lens[id * 32 + j]) and desc[id] =
// (na, m, ops, 0), or na = -1 when the pattern is not tiled.
void launch_tile_tab(int32_t npat, const int32_t *pat_canon, const int32_t *psteps,
                     const int32_t *a_rp, const int32_t *a_col, const int32_t *b_rp,
                     const int32_t *c_rp, const int64_t *moff, const uint16_t *map,
                     uint16_t *tab, uint16_t *lens, int4 *desc, cudaStream_t s);
// Tiles of the n rows (pid_of_row: pattern of each table row, -1 for the
// others): tiles[*ntiles] = (first row, lane mask, pattern, 0); the table rows
// no tile takes go to lo_rows / lo_ids (count *lo_n).  maxima (3 words,
// zeroed by the caller): stage floats, A segment entries and C row the tile
// kernel must hold.
void launch_tile_build(int32_t n, const int32_t *pid_of_row, const int4 *desc,
                       const uint16_t *lens, const int32_t *a_rp, const int32_t *a_col,
                       const int32_t *b_rp, const int32_t *c_rp, int4 *tiles, int32_t *ntiles,
                       int32_t *lo_rows, int32_t *lo_ids, int32_t *lo_n, int32_t *maxima,
                       cudaStream_t s);
// rows / ids (count at *count, zeroed by the caller): every row with
// pid_of_row[row] >= 0 and its pattern.
void launch_tile_list(int32_t n, const int32_t *pid_of_row, int32_t *rows, int32_t *ids,
                      int32_t *count, cudaStream_t s);
// Shared memory one warp of the tile kernel needs for those maxima.
size_t tile_smem_per_warp(int32_t stage_need, int32_t a_seg, int32_t max_out,
                          int32_t *acc_rows, int32_t *work_floats, int32_t *stage_cap);
// Values of the tiled rows (structure in C).
void launch_tile_numeric(const Operands &op, int32_t b_nnz, const int4 *tiles, int32_t ntiles,
                         const int4 *desc, const uint16_t *lens, const uint16_t *tab,
                         const int32_t *c_rp, float *c_val, int32_t stage_need, int32_t a_seg,
                         int32_t max_out, cudaStream_t s);

// ---- k_persist.cu ----------------------------------------------------------
// One persistent launch for the numeric-only pass of the merge and map rows
// of a plan (see k_persist.cu): the rows of each class cut into items of
// per_item rows, numbered from item0; segments heaviest class first.
constexpr int kPersistThreads = 256;
struct PersistSeg {
  const int32_t *rows;  // the class's row list (nullptr: rows 0.. in order)
  int32_t cls, count, per_item, item0;
};
struct PersistPlan {
  PersistSeg seg[kNumClasses];
  int32_t nseg = 0, n_items = 0;
};
// Classes the persistent kernel takes (merge and map classes).
bool persist_class(int cls);
// head: one int the launch clears first; max_map_out: the largest C row of
// the map classes in the plan (their accumulators).
void launch_persist_numeric(const Operands &op, const int64_t *ops, const PersistPlan &pp,
                            int32_t *head, const int32_t *c_rp, float *c_val,
                            const int64_t *moff, const uint16_t *map, int32_t *status,
                            int32_t max_map_out, int blocks_per_sm, int num_sms,
                            cudaStream_t s);

// ---- k_jit.cu --------------------------------------------------------------
// A nonzeros staged together by a pattern kernel: runs of at most this many.
constexpr int kJitMaxGroup = 8;
// One pattern for a compiled kernel (see k_jit.cu): na A nonzeros, B row
// lengths len[j], slot[t] = output position of flattened product t, m
// outputs, groups = [first, end) runs of A nonzeros whose B values are
// staged by one copy.
struct JitRequest {
  int na = 0, m = 0;
  int len[32] = {};
  std::vector<int> slot;
  std::vector<std::pair<int, int>> groups;
  void *kernel = nullptr;  // out: nullptr when NVRTC is missing or the compile failed
};
// Compiles the requests' kernels (side by side; cached for the process);
// returns how many compiled.
int jit_pattern_kernels(std::vector<JitRequest> &reqs);
void jit_stats(int32_t *compiles, double *ms);
// The groups of a pattern from its union spans (launch_jit_spans): runs of
// A nonzeros grown while the next one adds less than half its own span and
// the union stays within max_span floats.  *stage_need = the largest union.
std::vector<std::pair<int, int>> jit_groups(int na, const int *len, const int32_t *span,
                                            int32_t max_span, int32_t *stage_need);
// span[j0 * kJitMaxGroup + g - 1] = the largest B range (floats) that one of
// a sample of the tiles reads for A nonzeros j0 .. j0 + g - 1 (span zeroed by
// the caller; desc->x = the pattern's A nonzeros, nothing done unless in
// 1..32).
void launch_jit_spans(const int4 *tiles, int32_t ntiles, const int4 *desc, const uint16_t *lens,
                      const int32_t *a_rp, const int32_t *a_col, const int32_t *b_rp,
                      int32_t *span, int num_sms, cudaStream_t s);
// Marks pattern pid's tiles for the table kernel to skip (desc[pid].w = 1).
void launch_mark_pattern(int4 *desc, int32_t pid, cudaStream_t s);
// out[*n] = the tiles whose pattern is not marked (*n zeroed by the caller).
void launch_table_tiles(const int4 *tiles, int32_t ntiles, const int4 *desc, int4 *out,
                        int32_t *n, cudaStream_t s);
// Words of one tile record of a pattern kernel (na A nonzeros, ngroups
// staging groups).
int32_t jit_record_words(int na, int ngroups);
// The tile records of a pattern (see k_jit.cu): prog[ntiles * record words],
// arange[ntiles] = the A range of each tile, maxima[0] = the longest,
// maxima[1 + g] = group g's largest B range (zeroed by the caller);
// groups_dev = the groups as int2 on the device.
void launch_jit_programs(const int4 *tiles, int32_t ntiles, int32_t na,
                         const std::vector<std::pair<int, int>> &groups, const int2 *groups_dev,
                         const uint16_t *lens, const int32_t *a_rp, const int32_t *a_col,
                         const int32_t *b_rp, int32_t *prog, int2 *arange, int32_t *maxima,
                         int num_sms, cudaStream_t s);
// Shared memory of one warp of a pattern kernel, in floats: two tile buffers
// (record + A values) of *abuf_floats and two B stage buffers of *stage_cap
// (the largest B range `need` plus widening; room for 16 output rows).
void jit_layout(int32_t rw, int32_t seg_max, int32_t need, int32_t m, int32_t *stage_cap,
                int32_t *abuf_floats, int32_t *work_floats);
// Blocks of a persistent pattern kernel launch: the tiles' pairs, at most
// what fits the SMs at once.
int jit_grid(void *kernel, int32_t ntiles, int32_t work_floats, int32_t m, int num_sms);
// One launch of a pattern kernel over its tile records (head: one device
// word for the launch's tile queue, zeroed here; status: kDevWaitTimeout
// when a bounded wait ran out).
cudaError_t launch_pattern_kernel(void *kernel, const Operands &op, const int32_t *prog,
                                  const int2 *arange, int32_t ntiles, const int32_t *c_rp,
                                  float *c_val, int32_t stage_cap, int32_t abuf_floats,
                                  int32_t work_floats, int grid, int32_t *head,
                                  int32_t *status, cudaStream_t s);

// ---- k_shift.cu ------------------------------------------------------------
// Shift classes (see k_shift.cu).  Every pass but the probe is gated by the
// device flag *on, which the probe's decision sets, so the plan queues them
// without a host round trip.
int32_t shift_max_ops();
int32_t shift_samples();
// Keys and product counts of up to shift_samples() rows spread over A (keys:
// twice that many words) and the decision *on (1: at least half of them
// share their key and they average at least min_mean_ops products).
void launch_shift_decide(const Operands &op, unsigned long long *keys, int32_t min_mean_ops,
                         int32_t *on, CheckGuard guard, cudaStream_t s);
// bcls[b_rows], rcls[a_rows]: the class (smallest verified translate) of
// every B row and row; bkey / rkey / tkey / trow scratch, tcap a power of two
// >= 2 max(a_rows, b_rows).
void launch_shift_classes(const int32_t *on, const Operands &op, int32_t b_rows,
                          const int64_t *ops, unsigned long long *bkey,
                          unsigned long long *rkey, unsigned long long *tkey, int32_t *trow,
                          size_t tcap, int32_t *bcls, int32_t *rcls, cudaStream_t s);
// Patterns (classes of at least min_share rows whose canonical row has at
// most 512 outputs): pat_of[row] / pat_canon / pat_cap / pat_m (-1: dropped)
// / *npat (zeroed by the caller); members: pid_of_row[row] = their pattern
// (else -1; all -1 when *on is 0), cls[row] = empty, *members += count;
// class_count = the census of cls afterwards.
void launch_shift_patterns(const int32_t *on, const Operands &op, const int32_t *rcls,
                           int32_t *share, int32_t min_share, const int64_t *ops,
                           int32_t *pat_of, int32_t *pat_canon, int32_t *pat_cap,
                           int32_t *pat_m, int32_t *npat, int32_t cap_pat,
                           int32_t *pid_of_row, uint8_t *cls, int32_t *members,
                           int32_t *class_count, int num_sms, cudaStream_t s);
// counts[member] = counts[its canonical row].
void launch_shift_copy_counts(const int32_t *on, int32_t n, const int32_t *pid_of_row,
                              const int32_t *rcls, int32_t *counts, cudaStream_t s);
// Member rows' columns: the canonical row's moved by the row distance.
void launch_shift_fill(int32_t n, const int32_t *pid_of_row, const int32_t *rcls,
                       const int32_t *c_rp, int32_t *c_col, cudaStream_t s);
// Maps of the canonical rows (moff[canonical] = id * shift_max_ops()).
void launch_shift_canon_map(int32_t npat, const int32_t *pat_canon, const Operands &op,
                            const int32_t *c_rp, const int32_t *c_col, int64_t *moff,
                            uint16_t *map, cudaStream_t s);
// out[0] = largest products (rounded up to 32), out[1] = largest C row over
// the patterns with pat_m >= 0 (out zeroed by the caller).
void launch_pat_maxima(int32_t npat, const int32_t *pat_canon, const int32_t *pat_m,
                       const int64_t *ops, int32_t *out, cudaStream_t s);

// ---- k_check.cu ------------------------------------------------------------
// *result (initialised to ~0ull) receives min over bad rows of
// ((row + 1) << 8 | code); row -1 means row_ptr[0] != 0.  long_rows: scratch
// of 1 + check_long_rows_cap(rows, nnz) ints, long_rows[0] zeroed by the
// caller (the count of rows over 256 entries, listed after it).
int32_t check_long_rows_cap(int32_t rows, int32_t nnz);
void launch_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                      const int32_t *col_idx, int32_t nnz,
                      unsigned long long *result, int32_t *long_rows,
                      cudaStream_t s);

// ---- k_numeric.cu ----------------------------------------------------------
// Values (and, when fill, sorted columns) of the rows of one class.  With
// fo, the fused pass: rows go to their slab slots (c_col / c_val = slab),
// c_rp is unused and fill is implied.
void launch_numeric_class(int cls, const Operands &op, const int64_t *ops,
                          const int32_t *rows, int32_t nrows,
                          const int32_t *c_rp, int32_t *c_col, float *c_val,
                          bool fill, float *dense_acc, uint32_t *dense_bits,
                          int32_t dense_slots, int32_t *status, int num_sms,
                          cudaStream_t s, const FusedOut *fo = nullptr);
// Global scratch one dense numeric slot needs (accumulator + bitmap if the
// bitmap does not fit shared memory), 256-byte aligned.
size_t dense_slot_acc_bytes(int32_t b_cols);
size_t dense_slot_bits_bytes(int32_t b_cols);

// ---- k_mlp.cu ----------------------------------------------------------------
// Parameter layout of the 8 -> 32 -> 32 -> 2 row-binning MLP (floats):
// W1[32][8] b1[32] W2[32][32] b2[32] W3[2][32] b3[2] (trained), then the
// per-feature standardisation mean[8] and 1/sd[8] (set, not trained).
constexpr int kMlpIn = 8, kMlpHidden = 32, kMlpOut = 2;
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kMlpHidden * kMlpIn;
constexpr int kW2 = kB1 + kMlpHidden;
constexpr int kB2 = kW2 + kMlpHidden * kMlpHidden;
constexpr int kW3 = kB2 + kMlpHidden;
constexpr int kB3 = kW3 + kMlpOut * kMlpHidden;
constexpr int kMlpTrained = kB3 + kMlpOut;  // 1410
constexpr int kMu = kMlpTrained;
constexpr int kInvSd = kMu + kMlpIn;
constexpr int kMlpParams = kInvSd + kMlpIn;  // 1426
constexpr int kMlpParamsPad = (kMlpParams + 3) & ~3;

void launch_features(const Operands &op, float b_mean_len, float *feat,
                     int64_t *ops, int num_sms, cudaStream_t s);
// pred[row] = (y0, y1); ops (optional) = per-row op counts.
void launch_predict(const Operands &op, float b_mean_len, const float *params,
                    float2 *pred, int64_t *ops, int num_sms, cudaStream_t s);
// Learned binning for the fused pass: ops, class and slab capacity per row
// (counts[row] = 0 for empty rows) and rows per class.
void launch_learned_plan(const Operands &op, float b_mean_len, const float *params,
                         float scale, bool merge_ok, int64_t *ops, uint8_t *cls,
                         int32_t *cap, int32_t *counts, int32_t *class_count,
                         int num_sms, cudaStream_t s);
// grad (kMlpTrained floats, accumulated) and *loss_sum (accumulated) of the
// mean loss over n_total samples, for samples [0, n).
void launch_mlp_grad(const float *params, const float *feat, const float *target,
                     int32_t n, int32_t n_total, float *grad, float *loss_sum,
                     cudaStream_t s);
void launch_mlp_adam(float *params, const float *grad, float *m, float *v, float lr,
                     float b1, float b2, float eps, int step, cudaStream_t s);

}  // namespace rvsp
