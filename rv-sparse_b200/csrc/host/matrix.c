/*
 * Matrix lifecycle, status strings, host canonical check and the device
 * buffer helpers of the host layer.
 *
 * rvsp_csr_create / validate / destroy follow src/core/matrix.c:18-115 of
 * merledu/rv-sparse (same checks, same order, same codes); destroy also
 * frees device arrays owned by the library (owns_data == 2).  The status and
 * CSR-status strings are those of src/core/error.c:17-43 and
 * src/kernels/spgemm/rvsp_support.c:128-150.
 */
#include <limits.h>
#include <stdlib.h>
#include <string.h>

#include "rvsp_internal.h"

const char *rvsp_get_version(void)
{
    return "0.1.0";
}

const char *rvsp_status_to_string(rvsp_status_t status)
{
    switch (status) {
    case RVSP_SUCCESS:
        return "success";
    case RVSP_ERROR_NULL_POINTER:
        return "null pointer";
    case RVSP_ERROR_INVALID_ARGUMENT:
        return "invalid argument";
    case RVSP_ERROR_INVALID_CSR:
        return "invalid CSR matrix";
    case RVSP_ERROR_UNSUPPORTED_DTYPE:
        return "unsupported data type";
    case RVSP_ERROR_UNSUPPORTED_BACKEND:
        return "unsupported backend";
    case RVSP_ERROR_ALLOCATION_FAILED:
        return "allocation failed";
    case RVSP_ERROR_DEVICE:
        return "device error";
    default:
        return "unknown error";
    }
}

rvsp_status_t rvsp_csr_create(rvsp_csr_matrix_t *A, int32_t rows, int32_t cols,
                              int32_t nnz, int32_t *row_ptr, int32_t *col_idx,
                              void *values, rvsp_dtype_t dtype)
{
    if (!A || !row_ptr || !col_idx || !values)
        return RVSP_ERROR_NULL_POINTER;
    if (rows <= 0 || cols <= 0 || nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    A->rows = rows;
    A->cols = cols;
    A->nnz = nnz;
    A->row_ptr = row_ptr;
    A->col_idx = col_idx;
    A->values = values;
    A->dtype = dtype;
    A->format = RVSP_FORMAT_CSR;
    A->owns_data = 0;
    return rvsp_csr_validate(A);
}

rvsp_status_t rvsp_csr_validate(const rvsp_csr_matrix_t *A)
{
    if (!A || !A->row_ptr || !A->col_idx || !A->values)
        return RVSP_ERROR_NULL_POINTER;
    if (A->rows <= 0 || A->cols <= 0 || A->nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (A->row_ptr[0] != 0 || A->row_ptr[A->rows] != A->nnz)
        return RVSP_ERROR_INVALID_CSR;
    for (int32_t i = 0; i < A->rows; i++)
        if (A->row_ptr[i] > A->row_ptr[i + 1])
            return RVSP_ERROR_INVALID_CSR;
    for (int32_t i = 0; i < A->nnz; i++)
        if (A->col_idx[i] < 0 || A->col_idx[i] >= A->cols)
            return RVSP_ERROR_INVALID_CSR;
    return RVSP_SUCCESS;
}

void rvsp_csr_destroy(rvsp_csr_matrix_t *A)
{
    if (!A)
        return;
    if (A->owns_data == 1) {
        free(A->row_ptr);
        free(A->col_idx);
        free(A->values);
    } else if (A->owns_data == 2) {
        cudaFree(A->row_ptr);
        cudaFree(A->col_idx);
        cudaFree(A->values);
    }
    A->rows = 0;
    A->cols = 0;
    A->nnz = 0;
    A->row_ptr = NULL;
    A->col_idx = NULL;
    A->values = NULL;
    A->dtype = RVSP_DTYPE_FP32;
    A->format = RVSP_FORMAT_CSR;
    A->owns_data = 0;
}

rvsp_status_t rvsp_csr_copy_arrays(const rvsp_csr_matrix_t *src, rvsp_csr_matrix_t *dst)
{
    if (!src || !dst)
        return RVSP_ERROR_NULL_POINTER;
    if (src->rows != dst->rows || src->nnz != dst->nnz || src->rows < 0 || src->nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!src->row_ptr || !dst->row_ptr ||
        (src->nnz > 0 && (!src->col_idx || !src->values || !dst->col_idx || !dst->values)))
        return RVSP_ERROR_NULL_POINTER;
    cudaError_t e = cudaMemcpy(dst->row_ptr, src->row_ptr,
                               ((size_t)src->rows + 1) * sizeof(int32_t), cudaMemcpyDefault);
    if (e == cudaSuccess && src->nnz > 0)
        e = cudaMemcpy(dst->col_idx, src->col_idx, (size_t)src->nnz * sizeof(int32_t),
                       cudaMemcpyDefault);
    if (e == cudaSuccess && src->nnz > 0)
        e = cudaMemcpy(dst->values, src->values, (size_t)src->nnz * sizeof(float),
                       cudaMemcpyDefault);
    return rvsp_map_cuda(e);
}

rvsp_csr_status_t rvsp_csr_check(int32_t rows, int32_t cols,
                                 const int32_t *row_ptr,
                                 const int32_t *col_idx, int32_t *bad_row_out)
{
    if (bad_row_out)
        *bad_row_out = -1;
    if (rows < 0 || cols < 0 || row_ptr == NULL || row_ptr[0] != 0)
        return RVSP_CSR_BAD_ROW_PTR;
    for (int32_t r = 0; r < rows; r++) {
        const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
        rvsp_csr_status_t code = RVSP_CSR_OK;
        if (hi < lo) {
            code = RVSP_CSR_BAD_ROW_PTR;
        } else if (hi > lo) {
            if (col_idx == NULL)
                return RVSP_CSR_BAD_ROW_PTR; /* not row specific */
            int32_t last = -1;
            for (int32_t p = lo; p < hi && code == RVSP_CSR_OK; p++) {
                const int32_t c = col_idx[p];
                if (c < 0 || c >= cols)
                    code = RVSP_CSR_COL_OUT_OF_RANGE;
                else if (c == last)
                    code = RVSP_CSR_DUPLICATE;
                else if (c < last)
                    code = RVSP_CSR_UNSORTED;
                last = c;
            }
        }
        if (code != RVSP_CSR_OK) {
            if (bad_row_out)
                *bad_row_out = r;
            return code;
        }
    }
    return RVSP_CSR_OK;
}

const char *rvsp_csr_status_string(rvsp_csr_status_t status)
{
    switch (status) {
    case RVSP_CSR_OK:
        return "canonical CSR";
    case RVSP_CSR_BAD_ROW_PTR:
        return "malformed row pointer";
    case RVSP_CSR_COL_OUT_OF_RANGE:
        return "column index out of range";
    case RVSP_CSR_UNSORTED:
        return "column indices not ascending";
    case RVSP_CSR_DUPLICATE:
        return "duplicate column in row";
    default:
        return "unknown";
    }
}

rvsp_status_t rvsp_spgemm_buffer_size(int32_t b_cols, size_t *bytes_out)
{
    if (bytes_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (b_cols <= 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    /* The CUDA backend keeps its scratch on the device; a host-memory
     * descriptor compute() never touches the host workspace it is given. */
    *bytes_out = 256;
    return RVSP_SUCCESS;
}

/* ---- helpers ------------------------------------------------------------ */

rvsp_status_t rvsp_map_cuda(cudaError_t e)
{
    switch (e) {
    case cudaSuccess:
        return RVSP_SUCCESS;
    case cudaErrorMemoryAllocation:
        return RVSP_ERROR_ALLOCATION_FAILED;
    case cudaErrorNoDevice:
    case cudaErrorInsufficientDriver:
    case cudaErrorNoKernelImageForDevice:
    case cudaErrorInvalidDevice:
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    default:
        return RVSP_ERROR_DEVICE;
    }
}

rvsp_status_t rvsp_dbuf_reserve(rvsp_dbuf_t *b, size_t bytes)
{
    if (bytes == 0)
        bytes = 1;
    if (b->p && b->cap >= bytes)
        return RVSP_SUCCESS;
    if (b->p)
        cudaFree(b->p);
    b->p = NULL;
    b->cap = 0;
    cudaError_t e = cudaMalloc(&b->p, bytes);
    if (e != cudaSuccess) {
        b->p = NULL;
        cudaGetLastError();
        return rvsp_map_cuda(e);
    }
    b->cap = bytes;
    return RVSP_SUCCESS;
}

void rvsp_dbuf_release(rvsp_dbuf_t *b)
{
    if (b->p)
        cudaFree(b->p);
    b->p = NULL;
    b->cap = 0;
}

void rvsp_dev_csr_release(rvsp_dev_csr_t *d)
{
    rvsp_dbuf_release(&d->row_ptr);
    rvsp_dbuf_release(&d->col_idx);
    rvsp_dbuf_release(&d->values);
    d->h_row_ptr = NULL;
    d->h_col_idx = NULL;
    d->rows = 0;
    d->entries = 0;
}

rvsp_status_t rvsp_dev_csr_upload_structure(rvsp_dev_csr_t *d,
                                            const rvsp_csr_matrix_t *M,
                                            cudaStream_t s)
{
    const int32_t entries = M->row_ptr[M->rows];
    if (entries < 0)
        return RVSP_ERROR_INVALID_CSR;
    rvsp_status_t st =
        rvsp_dbuf_reserve(&d->row_ptr, ((size_t)M->rows + 1) * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&d->col_idx, (size_t)entries * sizeof(int32_t));
    if (st != RVSP_SUCCESS)
        return st;
    cudaError_t e = cudaMemcpyAsync(d->row_ptr.p, M->row_ptr,
                                    ((size_t)M->rows + 1) * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && entries > 0)
        e = cudaMemcpyAsync(d->col_idx.p, M->col_idx, (size_t)entries * sizeof(int32_t),
                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return rvsp_map_cuda(e);
    d->h_row_ptr = M->row_ptr;
    d->h_col_idx = M->col_idx;
    d->rows = M->rows;
    d->entries = entries;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_dev_csr_upload_values(rvsp_dev_csr_t *d,
                                         const rvsp_csr_matrix_t *M,
                                         cudaStream_t s)
{
    rvsp_status_t st =
        rvsp_dbuf_reserve(&d->values, (size_t)d->entries * sizeof(float));
    if (st != RVSP_SUCCESS)
        return st;
    if (d->entries > 0) {
        cudaError_t e = cudaMemcpyAsync(d->values.p, M->values,
                                        (size_t)d->entries * sizeof(float),
                                        cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
    }
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_device_check(rvsp_cuda_plan_t plan, cudaStream_t s,
                                int32_t rows, int32_t cols,
                                const int32_t *d_row_ptr,
                                const int32_t *d_col_idx, int32_t entries,
                                unsigned mask)
{
    int32_t code = 0, bad_row = -1;
    rvsp_status_t st = rvsp_cuda_csr_check(plan, s, rows, cols, d_row_ptr,
                                           d_col_idx, entries, &code, &bad_row);
    if (st != RVSP_SUCCESS)
        return st;
    if (code != 0 && (mask & (1u << (unsigned)code)))
        return RVSP_ERROR_INVALID_CSR;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_check_operand(const rvsp_csr_matrix_t *M)
{
    if (M == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (M->row_ptr == NULL || M->col_idx == NULL || M->values == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (M->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (M->rows <= 0 || M->cols <= 0 || M->nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return RVSP_SUCCESS;
}

rvsp_csr_status_t rvsp_csr_precheck(const rvsp_csr_matrix_t *M)
{
    if (M->rows < 0 || M->cols < 0 || M->row_ptr == NULL || M->row_ptr[0] != 0)
        return RVSP_CSR_BAD_ROW_PTR;
    if (M->col_idx == NULL) {
        for (int32_t r = 0; r < M->rows; r++) {
            if (M->row_ptr[r + 1] < M->row_ptr[r])
                return RVSP_CSR_BAD_ROW_PTR;
            if (M->row_ptr[r + 1] > M->row_ptr[r])
                return RVSP_CSR_BAD_ROW_PTR;
        }
    }
    if (M->cols == 0) {
        for (int32_t r = 0; r < M->rows; r++) {
            if (M->row_ptr[r + 1] < M->row_ptr[r])
                return RVSP_CSR_BAD_ROW_PTR;
            if (M->row_ptr[r + 1] > M->row_ptr[r])
                return RVSP_CSR_COL_OUT_OF_RANGE;
        }
    }
    return RVSP_CSR_OK;
}
