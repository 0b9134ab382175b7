/*
 * FP64 and INT8 -> INT32 one-shot products on the GPU: the CUDA form of the
 * reference's legacy scalar kernels, reached as in src/core/spgemm.c:179-193
 * (options {backend, FP64, FP64} and {backend, INT8, INT32}).
 *
 * Checks, in the order of the reference wrappers
 * (src/kernels/spgemm/legacy/csr_spgemm_wrappers.c):
 *   INT8: rvsp_csr_validate(A), (B) (:31-41); both INT8, else
 *         UNSUPPORTED_DTYPE (:43-46); A.cols == B.rows, else INVALID_ARGUMENT
 *         (:48-51); rows, cols and B's cols > 0, else INVALID_ARGUMENT
 *         (csr_scalar_i8.c:38-41).
 *   FP64: both FP64, else INVALID_ARGUMENT (:362-365); A.cols == B.rows, else
 *         INVALID_ARGUMENT (:367-370); negative sizes, bad row pointers or
 *         columns out of range give INVALID_ARGUMENT (csr_scalar_f64.c:57-138).
 * Then, unlike the legacy kernels (which accept unsorted rows), both operands
 * must be canonical: RVSP_ERROR_INVALID_CSR otherwise, since the GPU passes
 * rely on sorted, duplicate-free rows.
 *
 * Work: the FP32 path's symbolic pass and column fill give C's structure;
 * rvsp_cuda_typed_numeric computes the values in the reference's order;
 * rvsp_cuda_drop_zeros removes the entries equal to zero, as the legacy
 * kernels store only acc != 0.  C gets malloc'd host arrays (owns_data = 1),
 * dtype FP64 or INT32, as the reference wrappers set them.
 */
#include <stdlib.h>
#include <string.h>

#include "rvsp_internal.h"

static rvsp_status_t checks_f64(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B)
{
    if (A->dtype != RVSP_DTYPE_FP64 || B->dtype != RVSP_DTYPE_FP64)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (A->rows < 0 || A->cols < 0 || B->cols < 0 || !A->row_ptr || !A->col_idx ||
        !A->values || !B->row_ptr || !B->col_idx || !B->values)
        return RVSP_ERROR_INVALID_ARGUMENT;
    /* the legacy symbolic pass rejects bad row pointers and columns */
    const rvsp_csr_matrix_t *ops[2] = {A, B};
    for (int m = 0; m < 2; m++) {
        const rvsp_csr_matrix_t *M = ops[m];
        for (int32_t i = 0; i < M->rows; i++) {
            const int32_t s = M->row_ptr[i], e = M->row_ptr[i + 1];
            if (s < 0 || e < s)
                return RVSP_ERROR_INVALID_ARGUMENT;
            for (int32_t p = s; p < e; p++)
                if (M->col_idx[p] < 0 || M->col_idx[p] >= M->cols)
                    return RVSP_ERROR_INVALID_ARGUMENT;
        }
    }
    return RVSP_SUCCESS;
}

static rvsp_status_t checks_i8(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B)
{
    rvsp_status_t st = rvsp_csr_validate(A);
    if (st == RVSP_SUCCESS)
        st = rvsp_csr_validate(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->dtype != RVSP_DTYPE_INT8 || B->dtype != RVSP_DTYPE_INT8)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (A->rows <= 0 || A->cols <= 0 || B->cols <= 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return RVSP_SUCCESS;
}

static int canonical(const rvsp_csr_matrix_t *M)
{
    return rvsp_csr_check(M->rows, M->cols, M->row_ptr, M->col_idx, NULL) == RVSP_CSR_OK;
}

typedef struct {
    void *p[16];
    int n;
} dev_list_t;

static cudaError_t dalloc(dev_list_t *l, void **out, size_t bytes)
{
    if (l->n >= 16)
        return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(out, bytes ? bytes : 1);
    if (e == cudaSuccess)
        l->p[l->n++] = *out;
    return e;
}

static void dfree_all(dev_list_t *l)
{
    for (int i = 0; i < l->n; i++)
        cudaFree(l->p[i]);
    l->n = 0;
}

static cudaError_t upload(dev_list_t *l, void **out, const void *src, size_t bytes)
{
    cudaError_t e = dalloc(l, out, bytes);
    if (e == cudaSuccess && bytes)
        e = cudaMemcpy(*out, src, bytes, cudaMemcpyHostToDevice);
    return e;
}

rvsp_status_t rvsp_typed_oneshot(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                                 rvsp_csr_matrix_t *C, rvsp_dtype_t in_dtype)
{
    const int f64 = in_dtype == RVSP_DTYPE_FP64;
    rvsp_status_t st = f64 ? checks_f64(A, B) : checks_i8(A, B);
    if (st != RVSP_SUCCESS)
        return st;
    if (!canonical(A) || !canonical(B))
        return RVSP_ERROR_INVALID_CSR;
    const size_t in_sz = f64 ? sizeof(double) : sizeof(int8_t);
    const size_t out_sz = f64 ? sizeof(double) : sizeof(int32_t);
    const rvsp_dtype_t out_dtype = f64 ? RVSP_DTYPE_FP64 : RVSP_DTYPE_INT32;
    const int32_t a_nnz = A->row_ptr[A->rows], b_nnz = B->row_ptr[B->rows];
    if (A->rows == 0) { /* (FP64 only: INT8 requires rows > 0) an empty product */
        int32_t *rp = (int32_t *)calloc(1, sizeof(int32_t));
        int32_t *ci = (int32_t *)malloc(sizeof(int32_t));
        void *v = malloc(out_sz);
        if (!rp || !ci || !v) {
            free(rp);
            free(ci);
            free(v);
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        C->rows = 0;
        C->cols = B->cols;
        C->nnz = 0;
        C->row_ptr = rp;
        C->col_idx = ci;
        C->values = v;
        C->dtype = out_dtype;
        C->format = RVSP_FORMAT_CSR;
        C->owns_data = 1;
        return RVSP_SUCCESS;
    }

    dev_list_t l = {{0}, 0};
    rvsp_cuda_plan_t plan = NULL;
    void *a_rp = NULL, *a_ci = NULL, *a_v = NULL, *b_rp = NULL, *b_ci = NULL, *b_v = NULL;
    void *c_rp = NULL, *c_ci = NULL, *c_v = NULL, *ws = NULL;
    void *o_rp = NULL, *o_ci = NULL, *o_v = NULL;
    int32_t *h_rp = NULL, *h_ci = NULL;
    void *h_v = NULL;
    int64_t nnz = 0;
    int32_t kept = 0;
    cudaError_t e = cudaSuccess;

    st = rvsp_cuda_plan_create(&plan);
    if (st != RVSP_SUCCESS)
        return st;
    e = upload(&l, &a_rp, A->row_ptr, ((size_t)A->rows + 1) * sizeof(int32_t));
    if (e == cudaSuccess) e = upload(&l, &a_ci, A->col_idx, (size_t)a_nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = upload(&l, &a_v, A->values, (size_t)a_nnz * in_sz);
    if (e == cudaSuccess) e = upload(&l, &b_rp, B->row_ptr, ((size_t)B->rows + 1) * sizeof(int32_t));
    if (e == cudaSuccess) e = upload(&l, &b_ci, B->col_idx, (size_t)b_nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = upload(&l, &b_v, B->values, (size_t)b_nnz * in_sz);
    if (e == cudaSuccess) e = dalloc(&l, &c_rp, ((size_t)A->rows + 1) * sizeof(int32_t));
    if (e != cudaSuccess) {
        st = rvsp_map_cuda(e);
        goto done;
    }
    st = rvsp_cuda_symbolic(plan, NULL, A->rows, B->rows, B->cols, (const int32_t *)a_rp,
                            (const int32_t *)a_ci, (const int32_t *)b_rp,
                            (const int32_t *)b_ci, (int32_t *)c_rp, &nnz);
    if (st != RVSP_SUCCESS)
        goto done;
    {
        /* C's values buffer holds the fill's FP32 scratch values first
         * (4 bytes an entry; out_sz >= 4), then the typed sums. */
        const size_t ws_b = rvsp_cuda_numeric_workspace_bytes(plan);
        e = dalloc(&l, &c_ci, (size_t)nnz * sizeof(int32_t));
        if (e == cudaSuccess) e = dalloc(&l, &c_v, (size_t)nnz * out_sz);
        if (e == cudaSuccess && ws_b) e = dalloc(&l, &ws, ws_b);
        if (e != cudaSuccess) {
            st = rvsp_map_cuda(e);
            goto done;
        }
        /* The fill's columns do not depend on the values; A's and B's column
         * arrays stand in for FP32 values of the right length. */
        st = rvsp_cuda_numeric(plan, NULL, (const int32_t *)a_rp, (const int32_t *)a_ci,
                               (const float *)a_ci, (const int32_t *)b_rp,
                               (const int32_t *)b_ci, (const float *)b_ci,
                               (const int32_t *)c_rp, (int32_t *)c_ci, (float *)c_v, 1, ws,
                               ws_b);
        if (st != RVSP_SUCCESS)
            goto done;
    }
    e = cudaMemsetAsync(c_v, 0, (size_t)nnz * out_sz, NULL);
    if (e != cudaSuccess) {
        st = rvsp_map_cuda(e);
        goto done;
    }
    st = rvsp_cuda_typed_numeric(NULL, (int32_t)in_dtype, A->rows, (const int32_t *)a_rp,
                                 (const int32_t *)a_ci, a_v, (const int32_t *)b_rp,
                                 (const int32_t *)b_ci, b_v, (const int32_t *)c_rp,
                                 (const int32_t *)c_ci, c_v);
    if (st != RVSP_SUCCESS)
        goto done;
    e = dalloc(&l, &o_rp, ((size_t)A->rows + 1) * sizeof(int32_t));
    if (e == cudaSuccess) e = dalloc(&l, &o_ci, (size_t)nnz * sizeof(int32_t));
    if (e == cudaSuccess) e = dalloc(&l, &o_v, (size_t)nnz * out_sz);
    if (e != cudaSuccess) {
        st = rvsp_map_cuda(e);
        goto done;
    }
    st = rvsp_cuda_drop_zeros(NULL, (int32_t)out_dtype, A->rows, (const int32_t *)c_rp, nnz,
                              (const int32_t *)c_ci, c_v, (int32_t *)o_rp, (int32_t *)o_ci,
                              o_v, &kept);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_status(plan, NULL);
    if (st != RVSP_SUCCESS)
        goto done;
    {
        const size_t kn = (size_t)(kept > 0 ? kept : 1);
        h_rp = (int32_t *)malloc(((size_t)A->rows + 1) * sizeof(int32_t));
        h_ci = (int32_t *)malloc(kn * sizeof(int32_t));
        h_v = malloc(kn * out_sz);
        if (!h_rp || !h_ci || !h_v) {
            st = RVSP_ERROR_ALLOCATION_FAILED;
            goto done;
        }
        e = cudaMemcpy(h_rp, o_rp, ((size_t)A->rows + 1) * sizeof(int32_t),
                       cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && kept > 0)
            e = cudaMemcpy(h_ci, o_ci, (size_t)kept * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && kept > 0)
            e = cudaMemcpy(h_v, o_v, (size_t)kept * out_sz, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            st = rvsp_map_cuda(e);
            goto done;
        }
    }
    C->rows = A->rows;
    C->cols = B->cols;
    C->nnz = kept;
    C->row_ptr = h_rp;
    C->col_idx = h_ci;
    C->values = h_v;
    C->dtype = out_dtype;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = 1;
    h_rp = NULL;
    h_ci = NULL;
    h_v = NULL;
done:
    free(h_rp);
    free(h_ci);
    free(h_v);
    dfree_all(&l);
    rvsp_cuda_plan_destroy(plan);
    return st;
}
