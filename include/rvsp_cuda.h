/*
 * rv-sparse-b200: thin C-ABI layer over the sm_100a kernels.
 *
 * Plain C, raw DEVICE pointers and sizes, rvsp_status_t results.  The host
 * API (rv_sparse.h) is built on these calls; they are exported so a caller
 * that already keeps CSR arrays in device memory can drive the phases
 * directly, the way the reference's descriptor drives its kernel phases
 * (src/kernels/spgemm/rvsp_spgemm.h:56-121 in merledu/rv-sparse).
 *
 * A plan holds the analysis of one product between the phases: per-row op
 * counts, row classes and the rows of each class, all in device memory.  A
 * plan is not thread-safe; use one per host thread (or per stream).
 *
 * Streams: `stream` is a cudaStream_t (NULL = legacy default stream).  Calls
 * that must report a size to the host (symbolic) synchronize the stream;
 * numeric is asynchronous and its device status is read by
 * rvsp_cuda_plan_status.
 */
#ifndef RVSP_CUDA_H
#define RVSP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "rv_sparse_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rvsp_cuda_plan *rvsp_cuda_plan_t;

/* New: creates a plan on the current CUDA device.  UNSUPPORTED_BACKEND when
 * there is no usable sm_100 device. */
rvsp_status_t rvsp_cuda_plan_create(rvsp_cuda_plan_t *plan);

/* New.  NULL is accepted. */
void rvsp_cuda_plan_destroy(rvsp_cuda_plan_t plan);

/* Replaces rvsp_symbolic_count (rvsp_spgemm.h:62-70, rvsp_symbolic.c:13-86):
 * per-row op counts, exact per-row output nnz, exclusive scan into
 * c_row_ptr[0..a_rows] (device) and the int64 total.  ALLOCATION_FAILED when
 * the total exceeds INT32_MAX, as in the reference.  One host round trip
 * when every non-empty row falls in the merge classes (at most 16 A
 * nonzeros and 2048 products; under the automatic merge policy only when A
 * has at least 32768 rows), two otherwise.
 * Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_symbolic(rvsp_cuda_plan_t plan, void *stream,
                                 int32_t a_rows, int32_t b_rows, int32_t b_cols,
                                 const int32_t *a_row_ptr,
                                 const int32_t *a_col_idx,
                                 const int32_t *b_row_ptr,
                                 const int32_t *b_col_idx, int32_t *c_row_ptr,
                                 int64_t *c_nnz_out);

/* Device workspace bytes rvsp_cuda_numeric needs for the analysed product
 * (the dense accumulators of very long rows; 0 when there are none).  No
 * reference counterpart: rvsp_compute_ws_bytes (rvsp_common.h:81-90) sizes
 * the reference's host workspace. */
size_t rvsp_cuda_numeric_workspace_bytes(rvsp_cuda_plan_t plan);

/* rvsp_cuda_symbolic with the canonical-CSR check of A (and of B when
 * check_b != 0) folded in: the checks (rvsp_cuda_csr_check) are queued
 * before the row statistics, which read only A's a_nnz entries and B's
 * b_rows + 1 row pointers whatever the structure holds, and one host round
 * trip returns both the checks' verdicts and the class sizes.  A structure
 * that fails either check gives RVSP_ERROR_INVALID_CSR and no pass that
 * depends on it does any work: the passes queued before the verdict reaches
 * the host (the merge rows' count and the scan, when merge classes are on)
 * read the verdict on the device and return without reading the
 * structure or writing c_row_ptr; the plan is left unanalysed.  Otherwise
 * the same results as rvsp_cuda_symbolic, with one host round trip fewer
 * than calling the check first.  INVALID_ARGUMENT when a_cols != b_rows (as
 * the reference's shape check, spgemm_descr.c:185-188).  Synchronizes
 * `stream`. */
rvsp_status_t rvsp_cuda_symbolic_checked(rvsp_cuda_plan_t plan, void *stream, int32_t a_rows,
                                         int32_t a_cols, int32_t a_nnz, int32_t b_rows,
                                         int32_t b_cols, int32_t b_nnz,
                                         const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                         const int32_t *b_row_ptr, const int32_t *b_col_idx,
                                         int check_b, int32_t *c_row_ptr,
                                         int64_t *c_nnz_out);

/* Replaces rvsp_symbolic_fill (rvsp_spgemm.h:72-79) and
 * rvsp_spgemm_scalar_f32_numeric (rvsp_spgemm.h:93, gustavson_core_f32.inc:
 * 18-64): writes c_values and, when fill != 0, c_col_idx sorted within rows.
 * c_row_ptr must hold the analysed row pointers.  With fill == 0, c_col_idx
 * must already hold this product's structure.  workspace: device, at least
 * rvsp_cuda_numeric_workspace_bytes(plan).  Asynchronous. */
rvsp_status_t rvsp_cuda_numeric(rvsp_cuda_plan_t plan, void *stream,
                                const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                const float *a_values, const int32_t *b_row_ptr,
                                const int32_t *b_col_idx, const float *b_values,
                                const int32_t *c_row_ptr, int32_t *c_col_idx,
                                float *c_values, int fill, void *workspace,
                                size_t workspace_bytes);

/* Copies the analysed per-row op counts (int64, rvsp_spgemm_get_op_counts,
 * spgemm_descr.c:357-380) into host memory.  Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_op_counts(rvsp_cuda_plan_t plan, void *stream,
                                  int64_t *host_out, int32_t n);

/* Waits for `stream` and returns (and clears) the first error the kernels
 * recorded in the plan's device status word. */
rvsp_status_t rvsp_cuda_plan_status(rvsp_cuda_plan_t plan, void *stream);

/* Device canonical-CSR check (rvsp_csr_check, rvsp_support.c:37-126):
 * returns a rvsp_csr_status_t code (0 = canonical) in *code_out and the first
 * offending row (or -1) in *bad_row_out.  Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_csr_check(rvsp_cuda_plan_t plan, void *stream,
                                  int32_t rows, int32_t cols,
                                  const int32_t *row_ptr,
                                  const int32_t *col_idx, int32_t nnz,
                                  int32_t *code_out, int32_t *bad_row_out);

/* Per-phase device time.  When enabled, every phase the plan launches is
 * bracketed by CUDA events on its stream; times accumulate per rvsp_phase_t
 * and are resolved (waiting on the events) when read. */
rvsp_status_t rvsp_cuda_plan_set_profiling(rvsp_cuda_plan_t plan, int enable);
rvsp_status_t rvsp_cuda_plan_phase_times(rvsp_cuda_plan_t plan, double *ms_out,
                                         int64_t *launches_out, int32_t n,
                                         int reset);

/* Rows per class of the last analysis (symbolic classes in sym_out, numeric
 * classes in num_out; n entries each, see RowClass in the kernels). */
rvsp_status_t rvsp_cuda_plan_class_counts(rvsp_cuda_plan_t plan,
                                          int32_t *sym_out, int32_t *num_out,
                                          int32_t n);

/* ---- the row-binning model (new; no reference counterpart) --------------
 *
 * A small MLP, 8 row features -> 32 -> 32 -> 2 (ReLU), trained on the GPU by
 * hand-written forward/backward/Adam kernels.  Output 0 predicts
 * log2(1 + nnz of the output row), output 1 is the logit of the accumulator
 * class (1: the merge accumulator is faster for the row, 0: the warp hash).
 * The learned SpGEMM path uses it to size each row's hash table and to fuse
 * the symbolic and numeric passes.  Parameters (1426 floats): W1[32][8],
 * b1[32], W2[32][32], b2[32], W3[2][32], b3[2], then the per-feature mean[8]
 * and 1/sd[8] used to standardise the inputs (not trained).
 *
 * Features of A row i (log2(1 + x) each): nnz(A row), ops = sum |B row k|,
 * max |B row k|, ops / nnz, column span of the row's products, min(ops, span),
 * b_cols, mean |B row| of B.  (rvsp_mlp_t is declared in rv_sparse_types.h.) */

#define RVSP_MLP_NUM_FEATURES 8
#define RVSP_MLP_NUM_OUTPUTS 2
#define RVSP_MLP_NUM_PARAMS 1426

/* He-uniform weights from `seed`, zero biases, identity standardisation. */
rvsp_status_t rvsp_mlp_create(rvsp_mlp_t *model, uint64_t seed);
void rvsp_mlp_destroy(rvsp_mlp_t model);
int32_t rvsp_mlp_num_params(void);
/* Host copies of all RVSP_MLP_NUM_PARAMS parameters (n >= that). */
rvsp_status_t rvsp_mlp_get_params(rvsp_mlp_t model, float *host_out, int32_t n);
rvsp_status_t rvsp_mlp_set_params(rvsp_mlp_t model, const float *host_in, int32_t n);
/* Raw features of every A row into features_out (device, a_rows x 8,
 * row-major) and, when not NULL, the op counts (device int64). */
rvsp_status_t rvsp_mlp_features(void *stream, int32_t a_rows, int32_t b_rows,
                                int32_t b_cols, const int32_t *a_row_ptr,
                                const int32_t *a_col_idx, const int32_t *b_row_ptr,
                                const int32_t *b_col_idx, float *features_out,
                                int64_t *op_counts_out);
/* Mean loss over n samples (features: device n x 8 raw features; targets:
 * device n x 2) and its gradient with respect to the 1410 trained
 * parameters, copied to the host.  Synchronizes `stream`. */
rvsp_status_t rvsp_mlp_gradient(rvsp_mlp_t model, void *stream, const float *features,
                                const float *targets, int32_t n,
                                float *grad_host_out, float *loss_out);
/* Adam (beta 0.9 / 0.999) over `epochs` passes of contiguous mini-batches of
 * `batch` samples; loss_history (host, `epochs` floats, may be NULL) receives
 * each epoch's mean loss. */
rvsp_status_t rvsp_mlp_train(rvsp_mlp_t model, void *stream, const float *features,
                             const float *targets, int32_t n, int32_t batch,
                             int32_t epochs, float lr, float *loss_history);
/* Per-row outputs (device a_rows x 2) for the product A x B. */
rvsp_status_t rvsp_mlp_predict(rvsp_mlp_t model, void *stream, int32_t a_rows,
                               int32_t b_rows, int32_t b_cols,
                               const int32_t *a_row_ptr, const int32_t *a_col_idx,
                               const int32_t *b_row_ptr, const int32_t *b_col_idx,
                               float *pred_out);
rvsp_status_t rvsp_mlp_save(rvsp_mlp_t model, const char *path);
rvsp_status_t rvsp_mlp_load(rvsp_mlp_t model, const char *path);

/* Learned analysis: the GPU form of rvsp_symbolic_count
 * (rvsp_symbolic.c:13-86) for RVSP_SPGEMM_ALGO_CUDA_LEARNED.  The model
 * predicts each row's output nnz and accumulator class; each row gets a slab
 * slot of capacity min(ub, ceil(capacity_scale * predicted) + 16); one fused
 * pass computes every row's sorted columns and values into its slot; rows
 * that need more than their capacity are detected on the device and redone
 * by the plain two-pass path.  Results (c_row_ptr, *c_nnz_out, op counts)
 * are identical to rvsp_cuda_symbolic's; the following rvsp_cuda_numeric
 * with fill != 0 copies the slab into C, and recomputes the values only if
 * A's or B's values changed since (checked by a 64-bit fingerprint).
 * Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_learned_symbolic(
    rvsp_cuda_plan_t plan, rvsp_mlp_t model, void *stream, int32_t a_rows,
    int32_t b_rows, int32_t b_cols, const int32_t *a_row_ptr, const int32_t *a_col_idx,
    const float *a_values, int32_t a_nnz, const int32_t *b_row_ptr,
    const int32_t *b_col_idx, const float *b_values, int32_t b_nnz,
    float capacity_scale, int32_t *c_row_ptr, int64_t *c_nnz_out);

/* Rows the last learned analysis had to redo with the plain path. */
int32_t rvsp_cuda_plan_overflow_rows(rvsp_cuda_plan_t plan);

/* Which rows may use the thread-per-row merge accumulator (rows of at most
 * 16 A nonzeros and 2048 products): 0 automatic (when the matrix has at least
 * 32768 rows), 1 never, 2 whenever a row is eligible.  The autotuner uses 1
 * and 2 to time both accumulators on the same rows. */
rvsp_status_t rvsp_cuda_plan_set_merge_policy(rvsp_cuda_plan_t plan, int32_t policy);

/* Row tiles for numeric-only repeats (1, the default) or not (0).  The GPU
 * form of the reference's numeric-only compute (spgemm_descr.c:330-349) for
 * runs of consecutive rows that share one term pattern: a warp computes 32
 * such rows at once, one per lane (k_tile.cu).  0 keeps every such row on the
 * warp-per-row table kernel; the values are the same either way.  Enabling
 * after the reuse structures were built without tiles rebuilds them on the
 * next numeric-only call. */
rvsp_status_t rvsp_cuda_plan_set_row_tiles(rvsp_cuda_plan_t plan, int32_t enable);

/* Rows the row tiles of the current reuse structures compute (0 when there
 * are none or tiles are off). */
int32_t rvsp_cuda_plan_tiled_rows(rvsp_cuda_plan_t plan);

/* Persistent numeric-only pass (k_persist.cu): merge_rows > 0 (a multiple
 * of 32, at most 256) runs the numeric-only computes' merge-class and
 * map-class rows in one launch of blocks_per_sm (1..4) blocks per SM that
 * pull row bins (merge_rows merge rows, or 8 map rows, each) from a global
 * queue, heaviest class first; 0 (the default) keeps one launch per row
 * class.  The GPU form of the reference's numeric-only compute loop over rows
 * (spgemm_descr.c:330-349, gustavson_core_f32.inc:31-62); values are
 * identical either way.  The batch autotuner (rvsp_spgemm_batch_set_autotune)
 * times both. */
rvsp_status_t rvsp_cuda_plan_set_persistent(rvsp_cuda_plan_t plan, int32_t merge_rows,
                                           int32_t blocks_per_sm);

/* Pattern kernels (1, the default) or not (0).  When row tiles are built,
 * the (at most twelve) patterns with at least 128 tiles and at most 160
 * outputs a row get a kernel written for that pattern and compiled at run
 * time with NVRTC (k_jit.cu): persistent warps over per-tile records, each
 * lane keeping its row's outputs in registers, so a product is a shared
 * load, a multiply and an add.  Values are identical to the table kernel's
 * (same order, separately rounded products and sums).  Without NVRTC in the
 * process, or if a compile fails, the pattern stays on the table kernel.
 * Kernels are cached for the life of the process.  Changing the setting
 * rebuilds the tiles on the next numeric-only call.  A numeric-only call
 * runs its independent row groups on six internal streams of the plan,
 * forked from and joined back into the caller's stream. */
rvsp_status_t rvsp_cuda_plan_set_pattern_kernels(rvsp_cuda_plan_t plan, int32_t enable);

/* Rows (32 per tile, the tiles' masks not subtracted) the pattern kernels
 * of the current reuse structures take. */
int32_t rvsp_cuda_plan_pattern_kernel_rows(rvsp_cuda_plan_t plan);

/* Pattern kernels compiled in this process so far and the milliseconds the
 * compiles took (NULL outputs are skipped). */
void rvsp_cuda_pattern_kernel_stats(int32_t *compiles, double *compile_ms);

/* Shift classes in the analysis: 1 (the default) where they pay, 2 on any
 * matrix whose rows are translates, 0 never.  The GPU form of
 * rvsp_symbolic_count + rvsp_symbolic_fill (rvsp_symbolic.c:13-137) for rows
 * that are exact translates of another row (banded and stencil matrices):
 * such a row's A nonzeros sit at the same offsets from it as the other row's,
 * over B rows whose columns sit at the same offsets from their own index
 * (checked entry by entry).  Its count, columns (moved by the row distance)
 * and term table come from the canonical row, so it skips the symbolic pass
 * and the fill (k_shift.cu).  With 1, matrices of at least 32768 rows run a
 * probe of 2048 rows on the device, and the analysis only when at least half
 * of them have a translate among the others and they average at least 64
 * products (cheaper rows are left to the merge kernels: for them the
 * analysis and its tile builds cost more than one product saves); with 2,
 * any matrix of 64 rows or more whose sampled rows have translates.  The
 * learned analysis hands such matrices to it.  Values are identical either
 * way.  Applies from the next analysis. */
rvsp_status_t rvsp_cuda_plan_set_shift_classes(rvsp_cuda_plan_t plan, int32_t enable);

/* Rows of the last analysis that took their structure from a shift class (0
 * when none did). */
int32_t rvsp_cuda_plan_shift_rows(rvsp_cuda_plan_t plan);

/* Size of the library's fixed device scratch for rvsp_cuda_numeric_noalloc,
 * and the widest B it accepts (one float accumulator per B column). */
#define RVSP_NOALLOC_SCRATCH_BYTES (16u << 20)
#define RVSP_NOALLOC_MAX_B_COLS (RVSP_NOALLOC_SCRATCH_BYTES / 4u)

/* Numeric pass that allocates nothing.  No counterpart in the reference: its
 * CPU scalar backend takes a caller-allocated workspace, and every other
 * numeric entry point here takes a caller-allocated device workspace.  This
 * one is for callers that cannot call cudaMalloc when they need C's values:
 * memory pools and allocators that forbid re-entrant allocation from inside
 * their own callbacks, and latency-bound loops that must not take the
 * driver's allocation locks.
 *
 * Computes c_values for a structure (c_row_ptr, c_col_idx) that a symbolic
 * pass already produced for exactly this A and B; all pointers are device
 * pointers, the caller passes every input and output.  A and B must be
 * canonical CSR (as rvsp_cuda_csr_check accepts): column indices are
 * range-checked and skipped when out of range, row pointers are not, and a
 * B row that repeats a column races.  Values are bit-identical to
 * rvsp_cuda_numeric's.  Scratch is a fixed 16 MiB device array inside the
 * library (held by every GPU that loads it until the process exits).  The
 * first call on each device, with that device current, looks that array's
 * address up; make it before any stream capture.  Each call clears the
 * scratch it uses and is asynchronous on `stream`.  All calls share the one
 * array: calls that overlap on the GPU (different streams or host threads)
 * race, so serialise them.  a_rows == 0 or b_cols == 0 (an empty product)
 * returns RVSP_SUCCESS with no device work; a negative size, or
 * b_cols > RVSP_NOALLOC_MAX_B_COLS (4,194,304), is rejected with
 * RVSP_ERROR_INVALID_ARGUMENT before any device work; NULL pointers give
 * RVSP_ERROR_NULL_POINTER. */
rvsp_status_t rvsp_cuda_numeric_noalloc(void *stream, int32_t a_rows,
                                        int32_t b_rows, int32_t b_cols,
                                        const int32_t *a_row_ptr,
                                        const int32_t *a_col_idx,
                                        const float *a_values,
                                        const int32_t *b_row_ptr,
                                        const int32_t *b_col_idx,
                                        const float *b_values,
                                        const int32_t *c_row_ptr,
                                        const int32_t *c_col_idx,
                                        float *c_values);

/* Reuse map (no reference counterpart; the reference's numeric-only reuse,
 * spgemm_descr.c:330-351, reruns its dense accumulator).  Builds, for the
 * analysed structure already written into c_row_ptr / c_col_idx, the
 * position in C's row of every product of the warp-per-row rows (uint16 per
 * product, at most 24 GiB and a quarter of free device memory); later
 * rvsp_cuda_numeric calls with fill == 0 and this c_col_idx use it instead
 * of hashing C's columns.  rvsp_cuda_numeric builds it by itself on its first
 * numeric-only call outside stream capture; call this first when the repeats
 * will be captured.  *map_entries_out = products mapped (0 when the map does
 * not apply).  Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_plan_prepare_reuse(rvsp_cuda_plan_t plan, void *stream,
                                           const int32_t *a_row_ptr,
                                           const int32_t *a_col_idx,
                                           const int32_t *b_row_ptr,
                                           const int32_t *b_col_idx,
                                           const int32_t *c_row_ptr,
                                           const int32_t *c_col_idx,
                                           int64_t *map_entries_out);

/* Rows of the reuse map that read another row's identical map (a structured
 * matrix repeats a few position patterns over most rows; such rows share one
 * copy, found by fingerprint and confirmed entry by entry).  0 when no map
 * is built.  Synchronizes `stream`. */
rvsp_status_t rvsp_cuda_plan_reuse_shared_rows(rvsp_cuda_plan_t plan, void *stream,
                                               int32_t *shared_rows_out);

/* ---- FP64 and INT8 -> INT32 products ----------------------------------------
 * The values pass of the reference's legacy scalar kernels
 * (src/kernels/spgemm/legacy/csr_scalar_f64.c:196-262, csr_scalar_i8.c:
 * 137-185) for a structure already in c_row_ptr / c_col_idx (from
 * rvsp_cuda_symbolic and a fill by rvsp_cuda_numeric, whose columns do not
 * depend on the values).  in_dtype RVSP_DTYPE_FP64: double values, each entry
 * acc = fl(acc + fl(a * b)) over A's nonzeros in order from 0.0;
 * RVSP_DTYPE_INT8: int8 values, int32 sums of int32 products (wrapping).
 * c_values (double or int32, row_ptr[a_rows] entries) must be zeroed by the
 * caller.  Stream-ordered; other dtypes: RVSP_ERROR_UNSUPPORTED_DTYPE. */
rvsp_status_t rvsp_cuda_typed_numeric(void *stream, int32_t in_dtype, int32_t a_rows,
                                      const int32_t *a_row_ptr, const int32_t *a_col_idx,
                                      const void *a_values, const int32_t *b_row_ptr,
                                      const int32_t *b_col_idx, const void *b_values,
                                      const int32_t *c_row_ptr, const int32_t *c_col_idx,
                                      void *c_values);

/* Removes the entries equal to zero (the legacy kernels store only acc != 0;
 * -0.0 goes too), keeping row and column order: out_* receive the kept
 * entries (out arrays sized for nnz entries), *out_nnz their count.
 * out_dtype RVSP_DTYPE_FP64 (double values) or RVSP_DTYPE_INT32.  scratch:
 * device memory of rvsp_cuda_drop_zeros_scratch_bytes(nnz) bytes, 256-byte
 * aligned.  Synchronizes `stream` once (for the count), then leaves the
 * compaction queued on it. */
size_t rvsp_cuda_drop_zeros_scratch_bytes(int64_t nnz);
rvsp_status_t rvsp_cuda_drop_zeros(void *stream, int32_t out_dtype, int32_t rows,
                                   const int32_t *c_row_ptr, int64_t nnz,
                                   const int32_t *c_col_idx, const void *c_values,
                                   void *scratch, size_t scratch_bytes,
                                   int32_t *out_row_ptr, int32_t *out_col_idx,
                                   void *out_values, int32_t *out_nnz);

/* ---- Matrix Market ingest ------------------------------------------------
 * COO entries to canonical CSR on the device: the canonicalisation of the
 * reference's Matrix Market reader (tools/src/mtx_to_csr_formatter.c:67-146,
 * :214-311).  row / col / val: n device entries, 0-based, in file order.
 * symmetric != 0 appends the mirror (col, row, val) of every off-diagonal
 * entry after all stored entries, as the reference does.  Each row is sorted
 * by column; entries repeating a (row, column) are summed in that order from
 * the first (acc = v0, then acc = fl(acc + v)), so the result is the
 * reference's bit for bit.  c_row_ptr: device array of rows + 1, written.
 * *c_col_out / *c_val_out: device arrays of *c_nnz_out entries (at least
 * one), allocated here with cudaMalloc and owned by the caller (cudaFree).
 * An index outside [0, rows) x [0, cols) (or a mirror outside it) gives
 * RVSP_ERROR_INVALID_CSR (the reference does not check); more than
 * INT32_MAX output entries give RVSP_ERROR_ALLOCATION_FAILED.  Synchronizes
 * `stream`. */
rvsp_status_t rvsp_cuda_coo_to_csr(void *stream, int32_t rows, int32_t cols, int64_t n,
                                   int symmetric, const int32_t *row, const int32_t *col,
                                   const float *val, int32_t *c_row_ptr,
                                   int32_t **c_col_out, float **c_val_out,
                                   int32_t *c_nnz_out);

/* ---- Batches ------------------------------------------------------------
 * No reference counterpart: the reference computes one product per call.
 * A batch of independent products C_i = A_i * B_i is packed, a group of
 * products at a time, into one operand pair: A_g stacks the rows of the A_i
 * with each column index offset by the first row of B_i inside B_g, and B_g
 * stacks the rows of the B_i with their own column indices.  Row r of
 * A_g * B_g is then the matching row of its C_i, with the same terms in the
 * same order, and one symbolic and one numeric pass (one launch per row
 * class over the rows of every product) compute the whole group. */

/* One product, device pointers.  a_nnz / b_nnz are the entry counts
 * (row_ptr[rows]); rvsp_cuda_batch_entries fills them in. */
typedef struct {
    int32_t a_rows, b_rows, b_cols;
    int32_t a_nnz, b_nnz;
    const int32_t *a_row_ptr, *a_col_idx;
    const float *a_values;
    const int32_t *b_row_ptr, *b_col_idx;
    const float *b_values;
} rvsp_cuda_batch_item_t;

/* Where product i of a group starts inside A_g and B_g. */
typedef struct {
    int32_t a_row, a_nnz, b_row, b_nnz;
} rvsp_cuda_batch_offset_t;

/* items[i].a_nnz = a_row_ptr[a_rows] and items[i].b_nnz = b_row_ptr[b_rows]
 * for the `count` products of the device array `items`. */
rvsp_status_t rvsp_cuda_batch_entries(void *stream, rvsp_cuda_batch_item_t *items,
                                      int32_t count);

/* ops[i] += the products of item i (sum over A_i's nonzeros of the length of
 * the B_i row they select); *err |= 1 when an A_i column is not a B_i row
 * (that nonzero is skipped). */
rvsp_status_t rvsp_cuda_batch_op_counts(void *stream, const rvsp_cuda_batch_item_t *items,
                                        int32_t count, int64_t *ops, int32_t *err);

/* Packs the `count` products of `items` at offsets `off` into A_g and B_g:
 * structure and values when with_structure, values only otherwise.  *err
 * |= 2 / 4 for an A / B column out of range, 8 for a row_ptr[0] != 0. */
rvsp_status_t rvsp_cuda_batch_pack(void *stream, const rvsp_cuda_batch_item_t *items,
                                   const rvsp_cuda_batch_offset_t *off, int32_t count,
                                   int with_structure, int32_t *a_row_ptr,
                                   int32_t *a_col_idx, float *a_values,
                                   int32_t *b_row_ptr, int32_t *b_col_idx,
                                   float *b_values, int32_t *err);

/* Per-product views of C_g (row_ptr from 0):
 * c_rp_out[crp_off[i] + r] = c_row_ptr[off[i].a_row + r] -
 * c_row_ptr[off[i].a_row] for r = 0 .. a_rows, base_out[i] =
 * c_row_ptr[off[i].a_row] and nnz_out[i] = the product's nnz. */
rvsp_status_t rvsp_cuda_batch_views(void *stream, const rvsp_cuda_batch_item_t *items,
                                    const rvsp_cuda_batch_offset_t *off,
                                    const int64_t *crp_off, int32_t count,
                                    const int32_t *c_row_ptr, int32_t *c_rp_out,
                                    int32_t *base_out, int32_t *nnz_out);

#ifdef __cplusplus
}
#endif

#endif /* RVSP_CUDA_H */
