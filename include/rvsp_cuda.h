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
 * the total exceeds INT32_MAX, as in the reference.  Synchronizes `stream`. */
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

/* Size of the library's fixed device scratch for rvsp_cuda_numeric_noalloc,
 * and the widest B it accepts (one float accumulator per B column). */
#define RVSP_NOALLOC_SCRATCH_BYTES (16u << 20)
#define RVSP_NOALLOC_MAX_B_COLS (RVSP_NOALLOC_SCRATCH_BYTES / 4u)

/* Numeric pass that allocates nothing.  No counterpart in the reference: its
 * CPU scalar backend takes a caller-allocated workspace, and every other
 * numeric entry point here takes a caller-allocated device workspace.  This
 * one is for callers that cannot call cudaMalloc when they need C's values:
 * code running under CUDA graph capture, memory pools that forbid re-entrant
 * allocation, and latency-bound loops that must not take allocation locks.
 *
 * Computes c_values for a structure (c_row_ptr, c_col_idx) that a symbolic
 * pass already produced for this sparsity pattern; all pointers are device
 * pointers, the caller passes every input and output.  Values are
 * bit-identical to rvsp_cuda_numeric's.  Scratch is a fixed 16 MiB device
 * array inside the library (held by every GPU that loads it until the
 * process exits).  The first call on each device, with that device current,
 * looks that array's address up; make it before any stream capture.  Each
 * call clears the scratch it uses and is asynchronous on `stream`.  All calls
 * share the one array: calls that overlap on the GPU (different streams or
 * host threads) race, so serialise them.  b_cols > RVSP_NOALLOC_MAX_B_COLS
 * (4,194,304) is rejected with RVSP_ERROR_INVALID_ARGUMENT before any device
 * work; NULL pointers give RVSP_ERROR_NULL_POINTER. */
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

#ifdef __cplusplus
}
#endif

#endif /* RVSP_CUDA_H */
