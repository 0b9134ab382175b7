/*
 * Descriptor (two-phase) SpGEMM API on the CUDA backend.
 *
 * Same contract as src/core/spgemm_descr.c:19-380 of merledu/rv-sparse:
 *   - set_algo is refused after work_estimation (:102-125);
 *   - work_estimation discards any previous analysis, checks the operands
 *     (:137-160, :162-255) and reports the exact nnz(C) and a workspace size;
 *   - compute checks the descriptor state, the operands, their dimensions
 *     against the analysis, C's shape and capacity (:257-320), writes
 *     C.row_ptr, fills C.col_idx only when the analysed structure has not
 *     yet been written into this C->col_idx buffer (:330-341), then the
 *     values (:343-351);
 *   - get_op_counts returns int64 per row (:357-380);
 *   - invalidate_structure forces the next compute to refill (:129-135).
 *
 * The analysis (op counts, row classes, C.row_ptr) lives on the device in a
 * rvsp_cuda_plan.  In host memory space the descriptor also owns device
 * copies of A, B and C; in device memory space it copies nothing.
 */
#include <stdlib.h>
#include <string.h>

#include "rvsp_internal.h"

struct rvsp_spgemm_descr {
    rvsp_spgemm_algo_t algo;
    rvsp_memory_space_t mem;
    int estimated;

    cudaStream_t stream;     /* effective stream */
    cudaStream_t own_stream; /* created lazily when the caller gave none */
    int user_stream;
    int profiling;

    rvsp_cuda_plan_t plan;
    rvsp_mlp_t model;      /* learned algorithm only; not owned */
    float capacity_scale;  /* learned algorithm only */
    int32_t merge_policy;
    int32_t row_tiles;
    int32_t shift_classes;
    int32_t pattern_kernels;

    int32_t c_nnz;
    rvsp_dbuf_t c_row_ptr; /* analysed row pointers, device, a_rows + 1 */
    const int32_t *filled_into;

    int32_t a_rows, a_cols, a_nnz;
    int32_t b_rows, b_cols, b_nnz;
    size_t workspace_bytes;

    /* host memory space only */
    rvsp_dev_csr_t dA, dB;
    int b_aliases_a;
    rvsp_dbuf_t dC_col, dC_val, d_ws;
};

static int algo_supported(rvsp_spgemm_algo_t algo)
{
    return algo == RVSP_SPGEMM_ALGO_DEFAULT || algo == RVSP_SPGEMM_ALGO_CUDA_PLAIN ||
           algo == RVSP_SPGEMM_ALGO_CUDA_LEARNED;
}

rvsp_status_t rvsp_spgemm_descr_create(rvsp_spgemm_descr_t *descr)
{
    if (descr == NULL)
        return RVSP_ERROR_NULL_POINTER;
    *descr = NULL;
    struct rvsp_spgemm_descr *d =
        (struct rvsp_spgemm_descr *)rvsp_calloc(1, sizeof(*d));
    if (d == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    d->algo = RVSP_SPGEMM_ALGO_DEFAULT;
    d->mem = RVSP_MEM_HOST;
    d->capacity_scale = 1.15f;
    d->row_tiles = 1;
    d->shift_classes = 1;
    d->pattern_kernels = 1;
    *descr = d;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_model(rvsp_spgemm_descr_t d, rvsp_mlp_t model)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->model = model;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_capacity_scale(rvsp_spgemm_descr_t d, float scale)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!(scale > 0.0f) || scale > 1e6f)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->capacity_scale = scale;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_merge_policy(rvsp_spgemm_descr_t d, int32_t policy)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (d->estimated || policy < 0 || policy > 2)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->merge_policy = policy;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_row_tiles(rvsp_spgemm_descr_t d, int32_t enable)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (enable != 0 && enable != 1)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->row_tiles = enable;
    return d->plan ? rvsp_cuda_plan_set_row_tiles(d->plan, enable) : RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_shift_classes(rvsp_spgemm_descr_t d, int32_t enable)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (enable < 0 || enable > 2)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->shift_classes = enable;
    return d->plan ? rvsp_cuda_plan_set_shift_classes(d->plan, enable) : RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_pattern_kernels(rvsp_spgemm_descr_t d, int32_t enable)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (enable != 0 && enable != 1)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->pattern_kernels = enable;
    return d->plan ? rvsp_cuda_plan_set_pattern_kernels(d->plan, enable) : RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_shift_rows(rvsp_spgemm_descr_t d, int32_t *n_out)
{
    if (d == NULL || n_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    *n_out = d->plan ? rvsp_cuda_plan_shift_rows(d->plan) : 0;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_tiled_rows(rvsp_spgemm_descr_t d, int32_t *n_out)
{
    if (d == NULL || n_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    *n_out = d->plan ? rvsp_cuda_plan_tiled_rows(d->plan) : 0;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_overflow_rows(rvsp_spgemm_descr_t d, int32_t *n_out)
{
    if (d == NULL || n_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    *n_out = rvsp_cuda_plan_overflow_rows(d->plan);
    return RVSP_SUCCESS;
}

void rvsp_spgemm_descr_destroy(rvsp_spgemm_descr_t d)
{
    if (d == NULL)
        return;
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    rvsp_cuda_plan_destroy(d->plan);
    rvsp_dbuf_release(&d->c_row_ptr);
    rvsp_dev_csr_release(&d->dA);
    rvsp_dev_csr_release(&d->dB);
    rvsp_dbuf_release(&d->dC_col);
    rvsp_dbuf_release(&d->dC_val);
    rvsp_dbuf_release(&d->d_ws);
    if (d->own_stream)
        cudaStreamDestroy(d->own_stream);
    free(d);
}

rvsp_status_t rvsp_spgemm_set_algo(rvsp_spgemm_descr_t d, rvsp_spgemm_algo_t algo)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!algo_supported(algo))
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    d->algo = algo;
    return RVSP_SUCCESS;
}

void rvsp_spgemm_invalidate_structure(rvsp_spgemm_descr_t d)
{
    if (d != NULL)
        d->filled_into = NULL;
}

rvsp_status_t rvsp_spgemm_set_memory_space(rvsp_spgemm_descr_t d,
                                           rvsp_memory_space_t space)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (space != RVSP_MEM_HOST && space != RVSP_MEM_DEVICE)
        return RVSP_ERROR_INVALID_ARGUMENT;
    d->mem = space;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_stream(rvsp_spgemm_descr_t d, void *stream)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (stream) {
        d->stream = (cudaStream_t)stream;
        d->user_stream = 1;
    } else {
        d->stream = d->own_stream;
        d->user_stream = 0;
    }
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_set_profiling(rvsp_spgemm_descr_t d, int enable)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    d->profiling = enable != 0;
    if (d->plan)
        return rvsp_cuda_plan_set_profiling(d->plan, d->profiling);
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_phase_times(rvsp_spgemm_descr_t d, double *ms_out,
                                          int64_t *launches_out, int32_t n,
                                          int reset)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->plan) {
        for (int32_t i = 0; i < n; i++) {
            if (ms_out)
                ms_out[i] = 0.0;
            if (launches_out)
                launches_out[i] = 0;
        }
        return RVSP_SUCCESS;
    }
    return rvsp_cuda_plan_phase_times(d->plan, ms_out, launches_out, n, reset);
}

rvsp_status_t rvsp_spgemm_synchronize(rvsp_spgemm_descr_t d)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->plan)
        return RVSP_SUCCESS;
    return rvsp_cuda_plan_status(d->plan, d->stream);
}

/* Lazily creates the plan and the descriptor's own stream. */
static rvsp_status_t ensure_device(rvsp_spgemm_descr_t d)
{
    if (!d->plan) {
        rvsp_status_t st = rvsp_cuda_plan_create(&d->plan);
        if (st != RVSP_SUCCESS)
            return st;
        rvsp_cuda_plan_set_profiling(d->plan, d->profiling);
    }
    if (!d->own_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
    }
    if (!d->user_stream)
        d->stream = d->own_stream;
    rvsp_status_t st = rvsp_cuda_plan_set_row_tiles(d->plan, d->row_tiles);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_set_shift_classes(d->plan, d->shift_classes);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_set_pattern_kernels(d->plan, d->pattern_kernels);
    if (st != RVSP_SUCCESS)
        return st;
    return rvsp_cuda_plan_set_merge_policy(d->plan, d->merge_policy);
}

static int same_structure(const rvsp_csr_matrix_t *X, const rvsp_csr_matrix_t *Y)
{
    return X->row_ptr == Y->row_ptr && X->col_idx == Y->col_idx &&
           X->rows == Y->rows && X->cols == Y->cols;
}

/* Host memory space: brings the structure of A (and B unless B is A) to the
 * device when the host arrays differ from the ones uploaded, and checks it. */
static rvsp_status_t upload_structure(rvsp_spgemm_descr_t d,
                                      const rvsp_csr_matrix_t *A,
                                      const rvsp_csr_matrix_t *B, int force)
{
    rvsp_status_t st;
    if (force || d->dA.h_row_ptr != A->row_ptr || d->dA.h_col_idx != A->col_idx ||
        d->dA.rows != A->rows) {
        st = rvsp_dev_csr_upload_structure(&d->dA, A, d->stream);
        if (st != RVSP_SUCCESS)
            return st;
        st = rvsp_device_check(d->plan, d->stream, A->rows, A->cols,
                               (const int32_t *)d->dA.row_ptr.p,
                               (const int32_t *)d->dA.col_idx.p, d->dA.entries,
                               RVSP_REJECT_ALL);
        if (st != RVSP_SUCCESS)
            return st;
    }
    d->b_aliases_a = same_structure(A, B);
    if (!d->b_aliases_a &&
        (force || d->dB.h_row_ptr != B->row_ptr || d->dB.h_col_idx != B->col_idx ||
         d->dB.rows != B->rows)) {
        st = rvsp_dev_csr_upload_structure(&d->dB, B, d->stream);
        if (st != RVSP_SUCCESS)
            return st;
        st = rvsp_device_check(d->plan, d->stream, B->rows, B->cols,
                               (const int32_t *)d->dB.row_ptr.p,
                               (const int32_t *)d->dB.col_idx.p, d->dB.entries,
                               RVSP_REJECT_ALL);
        if (st != RVSP_SUCCESS)
            return st;
    }
    return RVSP_SUCCESS;
}

/* Host memory space: brings A's values (and B's, into their own array unless
 * B is A with the same values) to the device; *b_vals_out is B's device
 * values. */
static rvsp_status_t upload_values(rvsp_spgemm_descr_t d, const rvsp_csr_matrix_t *A,
                                   const rvsp_csr_matrix_t *B, const float **b_vals_out)
{
    cudaStream_t s = d->stream;
    rvsp_status_t st = rvsp_dev_csr_upload_values(&d->dA, A, s);
    const int b_values_alias = d->b_aliases_a && A->values == B->values;
    if (st == RVSP_SUCCESS && !d->b_aliases_a)
        st = rvsp_dev_csr_upload_values(&d->dB, B, s);
    if (st == RVSP_SUCCESS && d->b_aliases_a && !b_values_alias) {
        /* Same pattern, different values: B gets its own value array. */
        d->dB.entries = d->dA.entries;
        st = rvsp_dev_csr_upload_values(&d->dB, B, s);
    }
    *b_vals_out = (const float *)(b_values_alias ? d->dA.values.p : d->dB.values.p);
    return st;
}

rvsp_status_t rvsp_spgemm_work_estimation(rvsp_spgemm_descr_t d,
                                          const rvsp_csr_matrix_t *A,
                                          const rvsp_csr_matrix_t *B,
                                          size_t *workspace_bytes,
                                          int32_t *c_nnz_out)
{
    if (d == NULL || workspace_bytes == NULL || c_nnz_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    rvsp_status_t st = rvsp_check_operand(A);
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;

    /* Re-estimating discards any structure from a previous call. */
    d->estimated = 0;
    d->filled_into = NULL;
    d->c_nnz = 0;

    st = ensure_device(d);
    if (st != RVSP_SUCCESS)
        return st;

    const int32_t *a_rp, *a_ci, *b_rp, *b_ci;
    if (d->mem == RVSP_MEM_HOST) {
        st = upload_structure(d, A, B, 1);
        if (st != RVSP_SUCCESS)
            return st;
        a_rp = (const int32_t *)d->dA.row_ptr.p;
        a_ci = (const int32_t *)d->dA.col_idx.p;
        b_rp = d->b_aliases_a ? a_rp : (const int32_t *)d->dB.row_ptr.p;
        b_ci = d->b_aliases_a ? a_ci : (const int32_t *)d->dB.col_idx.p;
    } else {
        a_rp = A->row_ptr;
        a_ci = A->col_idx;
        b_rp = B->row_ptr;
        b_ci = B->col_idx;
        /* The plain path folds these checks into its symbolic pass (one host
         * round trip fewer, rvsp_cuda_symbolic_checked). */
        if (d->algo == RVSP_SPGEMM_ALGO_CUDA_LEARNED) {
            st = rvsp_device_check(d->plan, d->stream, A->rows, A->cols, a_rp, a_ci,
                                   A->nnz, RVSP_REJECT_ALL);
            if (st == RVSP_SUCCESS && !same_structure(A, B))
                st = rvsp_device_check(d->plan, d->stream, B->rows, B->cols, b_rp, b_ci,
                                       B->nnz, RVSP_REJECT_ALL);
            if (st != RVSP_SUCCESS)
                return st;
        }
    }

    st = rvsp_dbuf_reserve(&d->c_row_ptr, ((size_t)A->rows + 1) * sizeof(int32_t));
    if (st != RVSP_SUCCESS)
        return st;
    int64_t total = 0;
    if (d->algo == RVSP_SPGEMM_ALGO_CUDA_LEARNED) {
        if (d->model == NULL)
            return RVSP_ERROR_INVALID_ARGUMENT;
        /* The fused pass computes values too, so it needs them now.  The
         * value counts are those of the arrays on the device. */
        const float *a_v = (const float *)A->values, *b_v = (const float *)B->values;
        int32_t a_n = A->nnz, b_n = B->nnz;
        if (d->mem == RVSP_MEM_HOST) {
            st = upload_values(d, A, B, &b_v);
            if (st != RVSP_SUCCESS)
                return st;
            a_v = (const float *)d->dA.values.p;
            a_n = d->dA.entries;
            b_n = d->b_aliases_a ? d->dA.entries : d->dB.entries;
        }
        st = rvsp_cuda_learned_symbolic(d->plan, d->model, d->stream, A->rows, B->rows,
                                        B->cols, a_rp, a_ci, a_v, a_n, b_rp, b_ci, b_v,
                                        b_n, d->capacity_scale,
                                        (int32_t *)d->c_row_ptr.p, &total);
    } else if (d->mem == RVSP_MEM_DEVICE) {
        st = rvsp_cuda_symbolic_checked(d->plan, d->stream, A->rows, A->cols, A->nnz,
                                        B->rows, B->cols, B->nnz, a_rp, a_ci, b_rp, b_ci,
                                        !same_structure(A, B), (int32_t *)d->c_row_ptr.p,
                                        &total);
    } else {
        st = rvsp_cuda_symbolic(d->plan, d->stream, A->rows, B->rows, B->cols, a_rp,
                                a_ci, b_rp, b_ci, (int32_t *)d->c_row_ptr.p, &total);
    }
    if (st != RVSP_SUCCESS)
        return st;

    d->c_nnz = (int32_t)total;
    d->a_rows = A->rows;
    d->a_cols = A->cols;
    d->a_nnz = A->nnz;
    d->b_rows = B->rows;
    d->b_cols = B->cols;
    d->b_nnz = B->nnz;
    if (d->mem == RVSP_MEM_HOST) {
        rvsp_spgemm_buffer_size(B->cols, &d->workspace_bytes);
    } else {
        const size_t need = rvsp_cuda_numeric_workspace_bytes(d->plan);
        d->workspace_bytes = need > 256 ? need : 256;
    }
    d->estimated = 1;
    *workspace_bytes = d->workspace_bytes;
    *c_nnz_out = d->c_nnz;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_compute(rvsp_spgemm_descr_t d, const rvsp_csr_matrix_t *A,
                                  const rvsp_csr_matrix_t *B, rvsp_csr_matrix_t *C,
                                  void *workspace)
{
    if (d == NULL || C == NULL || workspace == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    rvsp_status_t st = rvsp_check_operand(A);
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->rows != d->a_rows || A->cols != d->a_cols || A->nnz != d->a_nnz ||
        B->rows != d->b_rows || B->cols != d->b_cols || B->nnz != d->b_nnz)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (C->row_ptr == NULL || C->col_idx == NULL || C->values == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (C->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (C->rows != d->a_rows || C->cols != d->b_cols)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (C->nnz < d->c_nnz)
        return RVSP_ERROR_INVALID_ARGUMENT;

    const int fill = d->filled_into != C->col_idx;
    const size_t nnz_c = (size_t)d->c_nnz;
    const size_t rp_bytes = ((size_t)d->a_rows + 1) * sizeof(int32_t);
    cudaStream_t s = d->stream;
    cudaError_t e;

    if (d->mem == RVSP_MEM_DEVICE) {
        e = cudaMemcpyAsync(C->row_ptr, d->c_row_ptr.p, rp_bytes,
                            cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
        st = rvsp_cuda_numeric(d->plan, s, A->row_ptr, A->col_idx,
                               (const float *)A->values, B->row_ptr, B->col_idx,
                               (const float *)B->values, C->row_ptr, C->col_idx,
                               (float *)C->values, fill, workspace,
                               d->workspace_bytes);
        if (st != RVSP_SUCCESS)
            return st;
    } else {
        st = upload_structure(d, A, B, 0);
        if (st != RVSP_SUCCESS)
            return st;
        const float *b_vals = NULL;
        st = upload_values(d, A, B, &b_vals);
        if (st != RVSP_SUCCESS)
            return st;
        const rvsp_dev_csr_t *bsrc = d->b_aliases_a ? &d->dA : &d->dB;
        st = rvsp_dbuf_reserve(&d->dC_col, nnz_c * sizeof(int32_t));
        if (st == RVSP_SUCCESS)
            st = rvsp_dbuf_reserve(&d->dC_val, nnz_c * sizeof(float));
        const size_t ws = rvsp_cuda_numeric_workspace_bytes(d->plan);
        if (st == RVSP_SUCCESS && ws > 0)
            st = rvsp_dbuf_reserve(&d->d_ws, ws);
        if (st != RVSP_SUCCESS)
            return st;
        st = rvsp_cuda_numeric(d->plan, s, (const int32_t *)d->dA.row_ptr.p,
                               (const int32_t *)d->dA.col_idx.p,
                               (const float *)d->dA.values.p,
                               (const int32_t *)bsrc->row_ptr.p,
                               (const int32_t *)bsrc->col_idx.p, b_vals,
                               (const int32_t *)d->c_row_ptr.p,
                               (int32_t *)d->dC_col.p, (float *)d->dC_val.p, fill,
                               ws > 0 ? d->d_ws.p : NULL, ws);
        if (st != RVSP_SUCCESS)
            return st;
        e = cudaMemcpyAsync(C->row_ptr, d->c_row_ptr.p, rp_bytes,
                            cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && fill && nnz_c > 0)
            e = cudaMemcpyAsync(C->col_idx, d->dC_col.p, nnz_c * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && nnz_c > 0)
            e = cudaMemcpyAsync(C->values, d->dC_val.p, nnz_c * sizeof(float),
                                cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
        st = rvsp_cuda_plan_status(d->plan, s);
        if (st != RVSP_SUCCESS)
            return st;
    }

    if (fill)
        d->filled_into = C->col_idx;
    C->nnz = d->c_nnz;
    C->format = RVSP_FORMAT_CSR;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_op_counts(rvsp_spgemm_descr_t d, int64_t *op_counts_out,
                                        int32_t n)
{
    if (d == NULL || op_counts_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (n < d->a_rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return rvsp_cuda_op_counts(d->plan, d->stream, op_counts_out, n);
}

rvsp_status_t rvsp_spgemm_get_class_counts(rvsp_spgemm_descr_t d, int32_t *sym_out,
                                           int32_t *num_out, int32_t n)
{
    if (d == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!d->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return rvsp_cuda_plan_class_counts(d->plan, sym_out, num_out, n);
}

rvsp_status_t rvsp_spgemm_multiply(rvsp_spgemm_descr_t d, const rvsp_csr_matrix_t *A,
                                   const rvsp_csr_matrix_t *B, rvsp_csr_matrix_t *C)
{
    if (d == NULL || A == NULL || B == NULL || C == NULL)
        return RVSP_ERROR_NULL_POINTER;
    size_t ws_bytes = 0;
    int32_t nnz = 0;
    rvsp_status_t st = rvsp_spgemm_work_estimation(d, A, B, &ws_bytes, &nnz);
    if (st != RVSP_SUCCESS)
        return st;
    const size_t alloc = (size_t)(nnz > 0 ? nnz : 1);
    const size_t rp_bytes = ((size_t)A->rows + 1) * sizeof(int32_t);
    rvsp_csr_matrix_t out;
    memset(&out, 0, sizeof(out));
    out.rows = A->rows;
    out.cols = B->cols;
    out.nnz = nnz;
    out.dtype = RVSP_DTYPE_FP32;
    out.format = RVSP_FORMAT_CSR;
    if (d->mem == RVSP_MEM_HOST) {
        out.owns_data = 1;
        out.row_ptr = (int32_t *)rvsp_malloc(rp_bytes);
        out.col_idx = (int32_t *)rvsp_malloc(alloc * sizeof(int32_t));
        out.values = rvsp_malloc(alloc * sizeof(float));
        void *ws = rvsp_malloc(ws_bytes > 0 ? ws_bytes : 1);
        if (!out.row_ptr || !out.col_idx || !out.values || !ws)
            st = RVSP_ERROR_ALLOCATION_FAILED;
        else
            st = rvsp_spgemm_compute(d, A, B, &out, ws);
        free(ws);
    } else {
        out.owns_data = 2;
        cudaError_t e = cudaMalloc((void **)&out.row_ptr, rp_bytes);
        if (e == cudaSuccess)
            e = cudaMalloc((void **)&out.col_idx, alloc * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMalloc(&out.values, alloc * sizeof(float));
        st = rvsp_map_cuda(e);
        if (st == RVSP_SUCCESS)
            st = rvsp_dbuf_reserve(&d->d_ws, ws_bytes);
        if (st == RVSP_SUCCESS)
            st = rvsp_spgemm_compute(d, A, B, &out, d->d_ws.p);
        if (st == RVSP_SUCCESS)
            st = rvsp_spgemm_synchronize(d);
    }
    if (st != RVSP_SUCCESS) {
        rvsp_csr_destroy(&out);
        C->row_ptr = NULL;
        C->col_idx = NULL;
        C->values = NULL;
        C->nnz = 0;
        C->owns_data = 0;
        return st;
    }
    *C = out;
    return RVSP_SUCCESS;
}
