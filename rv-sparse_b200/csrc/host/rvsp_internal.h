/*
 * Internal declarations shared by the host C files of rv-sparse-b200.
 */
#ifndef RVSP_INTERNAL_H
#define RVSP_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime_api.h>

#include "rv_sparse.h"
#include "rvsp_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A growable device buffer. */
typedef struct {
    void *p;
    size_t cap;
} rvsp_dbuf_t;

/* Host allocations of the library (alloc.c): malloc / calloc / realloc with
 * the failure hook of rvsp_debug.h; release with free(). */
void *rvsp_malloc(size_t n);
void *rvsp_calloc(size_t n, size_t size);
void *rvsp_realloc(void *p, size_t n);

rvsp_status_t rvsp_dbuf_reserve(rvsp_dbuf_t *b, size_t bytes);
void rvsp_dbuf_release(rvsp_dbuf_t *b);

rvsp_status_t rvsp_map_cuda(cudaError_t e);

/* Device copy of one CSR operand and the host arrays it mirrors. */
typedef struct {
    rvsp_dbuf_t row_ptr, col_idx, values;
    const void *h_row_ptr, *h_col_idx; /* structure currently uploaded */
    int32_t rows, entries;             /* entries = row_ptr[rows] */
} rvsp_dev_csr_t;

void rvsp_dev_csr_release(rvsp_dev_csr_t *d);

/* Uploads row_ptr and col_idx of a host CSR (entries = row_ptr[rows]). */
rvsp_status_t rvsp_dev_csr_upload_structure(rvsp_dev_csr_t *d,
                                            const rvsp_csr_matrix_t *M,
                                            cudaStream_t s);
rvsp_status_t rvsp_dev_csr_upload_values(rvsp_dev_csr_t *d,
                                         const rvsp_csr_matrix_t *M,
                                         cudaStream_t s);

/* Device canonical check of an uploaded operand: RVSP_SUCCESS when it passes
 * the checks in `mask` (bit c set = reject rvsp_csr_status_t c), else
 * RVSP_ERROR_INVALID_CSR. */
rvsp_status_t rvsp_device_check(rvsp_cuda_plan_t plan, cudaStream_t s,
                                int32_t rows, int32_t cols,
                                const int32_t *d_row_ptr,
                                const int32_t *d_col_idx, int32_t entries,
                                unsigned mask);

#define RVSP_REJECT_ALL 0x1Eu      /* BAD_ROW_PTR, RANGE, UNSORTED, DUPLICATE */

/* Reference check_operand (spgemm_descr.c:137-160). */
rvsp_status_t rvsp_check_operand(const rvsp_csr_matrix_t *M);

/* FP64 -> FP64 and INT8 -> INT32 one-shot products on the GPU (typed.c);
 * in_dtype RVSP_DTYPE_FP64 or RVSP_DTYPE_INT8. */
rvsp_status_t rvsp_typed_oneshot(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                                 rvsp_csr_matrix_t *C, rvsp_dtype_t in_dtype);

/* Host-side prefix of rvsp_csr_check that needs no column reads: negative
 * dims, NULL row_ptr, row_ptr[0] != 0, and (when col_idx is NULL) a
 * non-empty row.  Returns RVSP_CSR_OK when the device check must decide. */
rvsp_csr_status_t rvsp_csr_precheck(const rvsp_csr_matrix_t *M);

#ifdef __cplusplus
}
#endif

#endif
