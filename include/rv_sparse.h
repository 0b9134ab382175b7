/*
 * rv-sparse-b200: public API.
 *
 * Drop-in for the C API of merledu/rv-sparse (include/rv_sparse.h:27-142 in
 * that project).  Every reference function keeps its name, signature and
 * error behaviour; the comment above each cites the reference declaration it
 * replaces.  The additions below the reference API are marked "new".
 *
 * Backend.  This library computes FP32 CSR SpGEMM on one NVIDIA B200
 * (sm_100a) with hand-written CUDA kernels.  RVSP_BACKEND_CUDA is its only
 * backend; it has no CPU fallback.  A NULL options pointer selects it.
 *
 * Memory.  By default the descriptor API takes HOST arrays, exactly like the
 * reference: work_estimation and compute copy A and B to the device and C
 * back.  rvsp_spgemm_set_memory_space(descr, RVSP_MEM_DEVICE) switches a
 * descriptor to DEVICE pointers for A, B, C and the workspace, with no copies.
 *
 * Results.  C's structure (nnz, row_ptr, col_idx, ascending within rows) is
 * identical to the reference scalar backend's.  Each value accumulates its
 * terms in A's nonzero order with separately rounded multiply and add,
 * starting from +0.0f, so values are bit-identical to the scalar backend too.
 */
#ifndef RV_SPARSE_H
#define RV_SPARSE_H

#include <stddef.h>

#include "rv_sparse_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RVSP_VERSION_MAJOR 0
#define RVSP_VERSION_MINOR 1
#define RVSP_VERSION_PATCH 0

/* rv_sparse.h:27 */
const char *rvsp_get_version(void);

/* rv_sparse.h:29; also names RVSP_ERROR_DEVICE. */
const char *rvsp_status_to_string(rvsp_status_t status);

/* rv_sparse.h:38-46.  Wraps caller arrays without taking ownership, then
 * validates like rvsp_csr_validate.  Host arrays. */
rvsp_status_t rvsp_csr_create(rvsp_csr_matrix_t *A, int32_t rows, int32_t cols,
                              int32_t nnz, int32_t *row_ptr, int32_t *col_idx,
                              void *values, rvsp_dtype_t dtype);

/* rv_sparse.h:48.  Null arrays, dims, row_ptr[0] == 0, row_ptr[rows] == nnz,
 * non-decreasing row_ptr and column range; not sortedness.  Host arrays. */
rvsp_status_t rvsp_csr_validate(const rvsp_csr_matrix_t *A);

/* rv_sparse.h:50.  Frees host arrays when owns_data == 1, device arrays when
 * owns_data == 2, then resets the struct.  NULL is accepted. */
void rvsp_csr_destroy(rvsp_csr_matrix_t *A);

/* rv_sparse.h:63-67.  One-shot C = A * B on host arrays.  Checks canonical
 * CSR (RVSP_ERROR_INVALID_CSR), allocates C's host arrays (owns_data = 1)
 * and leaves C nulled on failure (spgemm.c:26-133). */
rvsp_status_t rvsp_spgemm_csr(const rvsp_csr_matrix_t *A,
                              const rvsp_csr_matrix_t *B,
                              rvsp_csr_matrix_t *C,
                              const rvsp_spgemm_options_t *options);

/* rv_sparse.h:81 */
rvsp_status_t rvsp_spgemm_descr_create(rvsp_spgemm_descr_t *descr);

/* rv_sparse.h:88.  NULL is accepted. */
void rvsp_spgemm_descr_destroy(rvsp_spgemm_descr_t descr);

/* rv_sparse.h:95-96.  Refused (INVALID_ARGUMENT) after work_estimation. */
rvsp_status_t rvsp_spgemm_set_algo(rvsp_spgemm_descr_t descr,
                                   rvsp_spgemm_algo_t algo);

/* rv_sparse.h:108-112.  Runs the symbolic analysis on the GPU; reports the
 * exact nnz(C) and the bytes of workspace compute() needs (host bytes in
 * host memory space, device bytes in device memory space). */
rvsp_status_t rvsp_spgemm_work_estimation(rvsp_spgemm_descr_t descr,
                                          const rvsp_csr_matrix_t *A,
                                          const rvsp_csr_matrix_t *B,
                                          size_t *workspace_bytes,
                                          int32_t *c_nnz_out);

/* rv_sparse.h:122-126.  Writes C.row_ptr, C.col_idx (only when the analysed
 * structure has not yet been written into this C->col_idx buffer) and
 * C.values.  Repeated calls with new values and the same pattern are
 * numeric-only. */
rvsp_status_t rvsp_spgemm_compute(rvsp_spgemm_descr_t descr,
                                  const rvsp_csr_matrix_t *A,
                                  const rvsp_csr_matrix_t *B,
                                  rvsp_csr_matrix_t *C, void *workspace);

/* rv_sparse.h:134-136.  Host int64 array of n >= rows entries. */
rvsp_status_t rvsp_spgemm_get_op_counts(rvsp_spgemm_descr_t descr,
                                        int64_t *op_counts_out, int32_t n);

/* rv_sparse.h:143.  NULL is accepted. */
void rvsp_spgemm_invalidate_structure(rvsp_spgemm_descr_t descr);

/* The reference also exports these helpers of its kernel layer
 * (src/kernels/spgemm/rvsp_spgemm.h:34-53); they are host functions here. */
typedef enum {
    RVSP_CSR_OK = 0,
    RVSP_CSR_BAD_ROW_PTR,
    RVSP_CSR_COL_OUT_OF_RANGE,
    RVSP_CSR_UNSORTED,
    RVSP_CSR_DUPLICATE
} rvsp_csr_status_t;

/* rvsp_spgemm.h:48-51.  Canonical-CSR check of host arrays, O(nnz). */
rvsp_csr_status_t rvsp_csr_check(int32_t rows, int32_t cols,
                                 const int32_t *row_ptr,
                                 const int32_t *col_idx, int32_t *bad_row_out);

/* rvsp_spgemm.h:53 */
const char *rvsp_csr_status_string(rvsp_csr_status_t status);

/* Matrix Market reader (no library counterpart: the reference's reader is
 * the tool function assemble_csr_matrix, tools/src/mtx_to_csr_formatter.c:
 * 148-325, returning vec_t arrays).  Reads a coordinate file into canonical
 * FP32 CSR the way that function does -- banner on the first line
 * ("pattern": values 1.0f; "symmetric": off-diagonal entries mirrored after
 * all stored ones), '%' lines skipped, "M N L", then up to L 1-based entries
 * read as fscanf reads them -- with the rows sorted by column and repeated
 * entries summed in file order on the GPU (rvsp_cuda_coo_to_csr); values are
 * the reference's bit for bit.  The text is parsed on all host cores.
 * space RVSP_MEM_HOST: host arrays (owns_data = 1); RVSP_MEM_DEVICE: device
 * arrays (owns_data = 2); free either with rvsp_csr_destroy.  cols = N.
 * Errors: unreadable file or size line -> RVSP_ERROR_INVALID_ARGUMENT; an
 * index outside 1..M x 1..N -> RVSP_ERROR_INVALID_CSR (the reference does
 * not check); no device -> RVSP_ERROR_UNSUPPORTED_BACKEND. */
rvsp_status_t rvsp_csr_read_mtx(const char *path, rvsp_memory_space_t space,
                                rvsp_csr_matrix_t *out);
/* The same on text already in memory (len bytes, need not end in NUL). */
rvsp_status_t rvsp_csr_parse_mtx(const char *text, size_t len, rvsp_memory_space_t space,
                                 rvsp_csr_matrix_t *out);

/* Copies the arrays of src into the arrays dst already holds (rows + 1 row
 * pointers, nnz columns and values; dst->rows and dst->nnz must equal
 * src's).  Either side may be host or device memory.  No reference
 * counterpart (its matrices live in host memory only). */
rvsp_status_t rvsp_csr_copy_arrays(const rvsp_csr_matrix_t *src, rvsp_csr_matrix_t *dst);

/* rvsp_spgemm.h:34.  Host workspace bytes of a descriptor compute() in host
 * memory space for a given b_cols. */
rvsp_status_t rvsp_spgemm_buffer_size(int32_t b_cols, size_t *bytes_out);

/* ---- new: device memory, streams, profiling ---------------------------- */

/* Selects host (default) or device pointers for A, B, C and the workspace.
 * Refused (INVALID_ARGUMENT) after work_estimation. */
rvsp_status_t rvsp_spgemm_set_memory_space(rvsp_spgemm_descr_t descr,
                                           rvsp_memory_space_t space);

/* Launches this descriptor's work on a caller-owned cudaStream_t (NULL: the
 * descriptor's own stream).  Calls still return only when their results are
 * complete, because estimation must report nnz(C). */
rvsp_status_t rvsp_spgemm_set_stream(rvsp_spgemm_descr_t descr, void *stream);

/* When enabled, each phase is bracketed by CUDA events on the launching
 * stream and its device time accumulates per rvsp_phase_t. */
rvsp_status_t rvsp_spgemm_set_profiling(rvsp_spgemm_descr_t descr, int enable);

/* Copies up to n accumulated phase times (ms) and launch counts (kernels
 * launched in that phase); either pointer may be NULL.  reset != 0 zeroes the
 * accumulators after reading. */
rvsp_status_t rvsp_spgemm_get_phase_times(rvsp_spgemm_descr_t descr,
                                          double *ms_out, int64_t *launches_out,
                                          int32_t n, int reset);

/* Device memory space: compute() is asynchronous with respect to the host
 * (stream-ordered).  This waits for the descriptor's stream and returns the
 * first error its kernels recorded (RVSP_ERROR_DEVICE), or RVSP_SUCCESS. */
rvsp_status_t rvsp_spgemm_synchronize(rvsp_spgemm_descr_t descr);

/* Rows per row class of the last analysis: symbolic classes (sized by the
 * op-count bound) in sym_out and numeric classes (sized by the exact row
 * nnz) in num_out, n entries each; either pointer may be NULL.  Classes in
 * order (12): empty; thread-per-row merge of at most 4 / 8 / 16 A nonzeros;
 * warp hash 64 / 128 / 256 / 512 / 1024 / 2048 slots; block 8192 (output
 * bound <= 4096); dense. */
rvsp_status_t rvsp_spgemm_get_class_counts(rvsp_spgemm_descr_t descr,
                                           int32_t *sym_out, int32_t *num_out,
                                           int32_t n);

/* ---- new: learned binning and single-call products -------------------- */

/* The row-binning model used by RVSP_SPGEMM_ALGO_CUDA_LEARNED (not owned;
 * keep it alive while the descriptor uses it).  work_estimation with the
 * learned algorithm and no model returns RVSP_ERROR_INVALID_ARGUMENT. */
rvsp_status_t rvsp_spgemm_set_model(rvsp_spgemm_descr_t descr, rvsp_mlp_t model);

/* Learned path: each row's slab capacity is
 * min(bound, ceil(scale * predicted nnz) + 16).  Default 1.15.  Smaller
 * values save slab memory and send more rows to the plain fallback. */
rvsp_status_t rvsp_spgemm_set_capacity_scale(rvsp_spgemm_descr_t descr, float scale);

/* Merge-accumulator policy of the descriptor's plan (see
 * rvsp_cuda_plan_set_merge_policy): 0 automatic, 1 never, 2 whenever
 * eligible.  Refused after work_estimation. */
rvsp_status_t rvsp_spgemm_set_merge_policy(rvsp_spgemm_descr_t descr, int32_t policy);

/* Row tiles for numeric-only computes (see rvsp_cuda_plan_set_row_tiles):
 * 1 (default) or 0.  Values are identical either way; allowed at any time. */
rvsp_status_t rvsp_spgemm_set_row_tiles(rvsp_spgemm_descr_t descr, int32_t enable);

/* Rows the row tiles compute in numeric-only computes (after the first
 * numeric-only compute on the current structure; 0 before). */
rvsp_status_t rvsp_spgemm_get_tiled_rows(rvsp_spgemm_descr_t descr, int32_t *n_out);

/* Pattern kernels for the row tiles (see rvsp_cuda_plan_set_pattern_kernels):
 * 1 (default) or 0.  Results are identical either way. */
rvsp_status_t rvsp_spgemm_set_pattern_kernels(rvsp_spgemm_descr_t descr, int32_t enable);

/* Shift classes in work_estimation (see rvsp_cuda_plan_set_shift_classes):
 * 1 (default: where they pay), 2 (whenever rows are translates) or 0.
 * Results are identical either way. */
rvsp_status_t rvsp_spgemm_set_shift_classes(rvsp_spgemm_descr_t descr, int32_t enable);

/* Rows of the last work_estimation that took their structure from a shift
 * class. */
rvsp_status_t rvsp_spgemm_get_shift_rows(rvsp_spgemm_descr_t descr, int32_t *n_out);

/* Rows the last learned work_estimation redid with the plain path. */
rvsp_status_t rvsp_spgemm_get_overflow_rows(rvsp_spgemm_descr_t descr, int32_t *n_out);

/* C = A * B in one call through the descriptor (its algorithm, memory space
 * and stream): work_estimation, allocation of C (host: malloc, owns_data =
 * 1; device: cudaMalloc, owns_data = 2) and compute.  With the learned
 * algorithm this is the fused single pass plus a copy into C. */
rvsp_status_t rvsp_spgemm_multiply(rvsp_spgemm_descr_t descr,
                                   const rvsp_csr_matrix_t *A,
                                   const rvsp_csr_matrix_t *B,
                                   rvsp_csr_matrix_t *C);

/* One-shot C = A * B with A, B and the resulting C in DEVICE memory.  C's
 * arrays are allocated with cudaMalloc and owns_data = 2. */
rvsp_status_t rvsp_spgemm_csr_device(const rvsp_csr_matrix_t *A,
                                     const rvsp_csr_matrix_t *B,
                                     rvsp_csr_matrix_t *C,
                                     const rvsp_spgemm_options_t *options);

/* ---- Batches (new; the reference computes one product per call) ---------
 *
 * Many independent products C_i = A_i * B_i of any sizes, computed together:
 *
 *   rvsp_spgemm_batch_create(&b);
 *   rvsp_spgemm_batch_add(b, &A_i, &B_i, &i);       for each product
 *   rvsp_spgemm_batch_work_estimation(b, &nnz);     structure of every C_i
 *   rvsp_spgemm_batch_compute(b);                   columns and values
 *   ... change the values of the A_i / B_i in place ...
 *   rvsp_spgemm_batch_compute(b);                   values only (graph replay)
 *   rvsp_spgemm_batch_get_result(b, i, &C_i);       device view of C_i
 *   rvsp_spgemm_batch_destroy(b);
 *
 * The batch keeps the A_i / B_i structs given to add (not copies of their
 * arrays): their arrays must stay valid, with unchanged structure, until
 * destroy; their values may change between computes.  Host memory space
 * (the default) takes host arrays; RVSP_MEM_DEVICE takes device arrays.
 *
 * work_estimation checks every operand (RVSP_ERROR_INVALID_CSR as
 * rvsp_spgemm_work_estimation does), packs the products into groups of at
 * most INT32_MAX intermediate products (multiply-adds) each, which keeps
 * every group's nnz(C) in int32, and runs one symbolic pass per group; every
 * row class is one launch over the rows of every product of the group.  The
 * first compute fills columns and values; every later compute is a
 * numeric-only repeat, captured into a CUDA graph on its first run and
 * replayed after.  Results are bit-identical to computing each product on
 * its own.  With autotune on, work_estimation times the merge-accumulator
 * policies (automatic, never, always) on the batch's own rows and keeps the
 * fastest, then times the numeric-only pass as one launch per row class and
 * as the persistent pass (rvsp_cuda_plan_set_persistent) with several bin
 * sizes and occupancies, and keeps the fastest shape. */
typedef struct rvsp_spgemm_batch *rvsp_spgemm_batch_t;

rvsp_status_t rvsp_spgemm_batch_create(rvsp_spgemm_batch_t *batch);
void rvsp_spgemm_batch_destroy(rvsp_spgemm_batch_t batch);
/* Before the first add. */
rvsp_status_t rvsp_spgemm_batch_set_memory_space(rvsp_spgemm_batch_t batch,
                                                 rvsp_memory_space_t space);
/* cudaStream_t for all device work of the batch (NULL: its own stream). */
rvsp_status_t rvsp_spgemm_batch_set_stream(rvsp_spgemm_batch_t batch, void *stream);
rvsp_status_t rvsp_spgemm_batch_set_autotune(rvsp_spgemm_batch_t batch, int enable);
rvsp_status_t rvsp_spgemm_batch_set_merge_policy(rvsp_spgemm_batch_t batch, int32_t policy);
/* Numeric-only shape of the batch's repeats (see rvsp_cuda_plan_set_persistent):
 * merge_rows 0 for one launch per row class, else merge rows per bin of the
 * persistent pass (a multiple of 32, at most 256), with blocks_per_sm 1..4.
 * Before work_estimation; autotune overrides it. */
rvsp_status_t rvsp_spgemm_batch_set_persistent(rvsp_spgemm_batch_t batch, int32_t merge_rows,
                                               int32_t blocks_per_sm);
/* The tuning in use: merge policy, persistent merge rows (0: per-class
 * launches) and blocks per SM; with autotune, the numeric-only milliseconds
 * of each shape tried (shape_ms_out: at least 8 floats, in the order
 * per-class, 128x2, 256x2, 256x1, 64x4) and their count.  NULL outputs are
 * skipped. */
rvsp_status_t rvsp_spgemm_batch_get_tuning(rvsp_spgemm_batch_t batch, int32_t *merge_policy_out,
                                           int32_t *merge_rows_out, int32_t *blocks_out,
                                           float *shape_ms_out, int32_t *n_shapes_out);
/* Largest op count of one group (default INT32_MAX; smaller values split a
 * batch into more groups). */
rvsp_status_t rvsp_spgemm_batch_set_group_ops(rvsp_spgemm_batch_t batch, int64_t max_ops);
/* Refused after work_estimation (RVSP_ERROR_INVALID_ARGUMENT); A->cols must
 * equal B->rows, both FP32. */
rvsp_status_t rvsp_spgemm_batch_add(rvsp_spgemm_batch_t batch, const rvsp_csr_matrix_t *A,
                                    const rvsp_csr_matrix_t *B, int32_t *index_out);
rvsp_status_t rvsp_spgemm_batch_work_estimation(rvsp_spgemm_batch_t batch,
                                                int64_t *total_nnz_out);
rvsp_status_t rvsp_spgemm_batch_compute(rvsp_spgemm_batch_t batch);
/* Waits for the batch's work and reports device-side errors. */
rvsp_status_t rvsp_spgemm_batch_synchronize(rvsp_spgemm_batch_t batch);
rvsp_status_t rvsp_spgemm_batch_get_nnz(rvsp_spgemm_batch_t batch, int32_t index,
                                        int32_t *nnz_out);
/* C_i as a CSR of DEVICE arrays owned by the batch (owns_data = 0), valid
 * until the next work_estimation or destroy; values are current after the
 * last compute. */
rvsp_status_t rvsp_spgemm_batch_get_result(rvsp_spgemm_batch_t batch, int32_t index,
                                           rvsp_csr_matrix_t *C_out);
/* Copies C_i into the caller's HOST arrays of C (row_ptr of rows + 1
 * entries, col_idx and values of at least nnz); synchronizes. */
rvsp_status_t rvsp_spgemm_batch_copy_result(rvsp_spgemm_batch_t batch, int32_t index,
                                            rvsp_csr_matrix_t *C);
/* Groups, total products (op count), the merge policy in use and the nodes
 * of the numeric-only graph (0 before its first capture); NULL outputs are
 * skipped. */
rvsp_status_t rvsp_spgemm_batch_get_stats(rvsp_spgemm_batch_t batch, int32_t *groups_out,
                                          int64_t *ops_out, int32_t *merge_policy_out,
                                          int32_t *graph_nodes_out);

#ifdef __cplusplus
}
#endif

#endif /* RV_SPARSE_H */
