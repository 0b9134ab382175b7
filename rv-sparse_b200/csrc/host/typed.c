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
#include <pthread.h>
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

/* Per-thread device context of the typed one-shot path: a plan, a stream and
 * grow-only device buffers, kept between calls so repeated products pay no
 * cudaMalloc / cudaFree; released when the thread exits. */
typedef struct {
    rvsp_cuda_plan_t plan;
    cudaStream_t stream;
    rvsp_dbuf_t a_rp, a_ci, a_v, b_rp, b_ci, b_v, c_rp, c_ci, c_v, ws, o_rp, o_ci, o_v, dz;
} typed_ctx_t;

static pthread_key_t g_typed_key;
static pthread_once_t g_typed_once = PTHREAD_ONCE_INIT;

static void typed_ctx_free(void *p)
{
    typed_ctx_t *c = (typed_ctx_t *)p;
    if (!c)
        return;
    if (c->stream)
        cudaStreamSynchronize(c->stream);
    rvsp_cuda_plan_destroy(c->plan);
    rvsp_dbuf_t *bufs[] = {&c->a_rp, &c->a_ci, &c->a_v, &c->b_rp, &c->b_ci, &c->b_v, &c->c_rp,
                           &c->c_ci, &c->c_v, &c->ws, &c->o_rp, &c->o_ci, &c->o_v, &c->dz};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        rvsp_dbuf_release(bufs[i]);
    if (c->stream)
        cudaStreamDestroy(c->stream);
    free(c);
}

static void typed_key_init(void) { pthread_key_create(&g_typed_key, typed_ctx_free); }

static rvsp_status_t typed_ctx(typed_ctx_t **out)
{
    pthread_once(&g_typed_once, typed_key_init);
    typed_ctx_t *c = (typed_ctx_t *)pthread_getspecific(g_typed_key);
    if (!c) {
        c = (typed_ctx_t *)rvsp_calloc(1, sizeof(*c));
        if (!c)
            return RVSP_ERROR_ALLOCATION_FAILED;
        rvsp_status_t st = rvsp_cuda_plan_create(&c->plan);
        if (st != RVSP_SUCCESS) {
            free(c);
            return st;
        }
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            rvsp_cuda_plan_destroy(c->plan);
            free(c);
            return rvsp_map_cuda(e);
        }
        pthread_setspecific(g_typed_key, c);
    }
    *out = c;
    return RVSP_SUCCESS;
}

static rvsp_status_t put(rvsp_dbuf_t *b, const void *src, size_t bytes, cudaStream_t s)
{
    rvsp_status_t st = rvsp_dbuf_reserve(b, bytes);
    if (st == RVSP_SUCCESS && bytes)
        st = rvsp_map_cuda(cudaMemcpyAsync(b->p, src, bytes, cudaMemcpyHostToDevice, s));
    return st;
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
    const size_t rp_b = ((size_t)A->rows + 1) * sizeof(int32_t);
    int32_t *h_rp = NULL, *h_ci = NULL;
    void *h_v = NULL;
    if (A->rows == 0) { /* (FP64 only: INT8 requires rows > 0) an empty product */
        h_rp = (int32_t *)rvsp_calloc(1, sizeof(int32_t));
        h_ci = (int32_t *)rvsp_malloc(sizeof(int32_t));
        h_v = rvsp_malloc(out_sz);
        if (!h_rp || !h_ci || !h_v) {
            st = RVSP_ERROR_ALLOCATION_FAILED;
            goto done;
        }
        goto out;
    }
    typed_ctx_t *c = NULL;
    st = typed_ctx(&c);
    if (st != RVSP_SUCCESS)
        return st;
    cudaStream_t s = c->stream;
    const int b_is_a = A->row_ptr == B->row_ptr && A->col_idx == B->col_idx &&
                       A->values == B->values && A->rows == B->rows;
    st = put(&c->a_rp, A->row_ptr, rp_b, s);
    if (st == RVSP_SUCCESS) st = put(&c->a_ci, A->col_idx, (size_t)a_nnz * sizeof(int32_t), s);
    if (st == RVSP_SUCCESS) st = put(&c->a_v, A->values, (size_t)a_nnz * in_sz, s);
    if (st == RVSP_SUCCESS && !b_is_a) {
        st = put(&c->b_rp, B->row_ptr, ((size_t)B->rows + 1) * sizeof(int32_t), s);
        if (st == RVSP_SUCCESS) st = put(&c->b_ci, B->col_idx, (size_t)b_nnz * sizeof(int32_t), s);
        if (st == RVSP_SUCCESS) st = put(&c->b_v, B->values, (size_t)b_nnz * in_sz, s);
    }
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->c_rp, rp_b);
    if (st != RVSP_SUCCESS)
        goto done;
    const int32_t *d_brp = (const int32_t *)(b_is_a ? c->a_rp.p : c->b_rp.p);
    const int32_t *d_bci = (const int32_t *)(b_is_a ? c->a_ci.p : c->b_ci.p);
    const void *d_bv = b_is_a ? c->a_v.p : c->b_v.p;
    int64_t nnz = 0;
    st = rvsp_cuda_symbolic(c->plan, s, A->rows, B->rows, B->cols, (const int32_t *)c->a_rp.p,
                            (const int32_t *)c->a_ci.p, d_brp, d_bci, (int32_t *)c->c_rp.p,
                            &nnz);
    if (st != RVSP_SUCCESS)
        goto done;
    /* C's values buffer holds the fill's FP32 scratch values first (4 bytes
     * an entry; out_sz >= 4), then the typed sums. */
    const size_t ws_b = rvsp_cuda_numeric_workspace_bytes(c->plan);
    const size_t dz_b = rvsp_cuda_drop_zeros_scratch_bytes(nnz);
    st = rvsp_dbuf_reserve(&c->c_ci, (size_t)nnz * sizeof(int32_t));
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->c_v, (size_t)nnz * out_sz);
    if (st == RVSP_SUCCESS && ws_b) st = rvsp_dbuf_reserve(&c->ws, ws_b);
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->o_rp, rp_b);
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->o_ci, (size_t)nnz * sizeof(int32_t));
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->o_v, (size_t)nnz * out_sz);
    if (st == RVSP_SUCCESS) st = rvsp_dbuf_reserve(&c->dz, dz_b);
    if (st != RVSP_SUCCESS)
        goto done;
    /* The fill's columns do not depend on the values; A's and B's column
     * arrays stand in for FP32 values of the right length. */
    st = rvsp_cuda_numeric(c->plan, s, (const int32_t *)c->a_rp.p, (const int32_t *)c->a_ci.p,
                           (const float *)c->a_ci.p, d_brp, d_bci, (const float *)d_bci,
                           (const int32_t *)c->c_rp.p, (int32_t *)c->c_ci.p,
                           (float *)c->c_v.p, 1, ws_b ? c->ws.p : NULL, ws_b);
    if (st == RVSP_SUCCESS)
        st = rvsp_map_cuda(cudaMemsetAsync(c->c_v.p, 0, (size_t)nnz * out_sz, s));
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_typed_numeric(s, (int32_t)in_dtype, A->rows, (const int32_t *)c->a_rp.p,
                                     (const int32_t *)c->a_ci.p, c->a_v.p, d_brp, d_bci, d_bv,
                                     (const int32_t *)c->c_rp.p, (const int32_t *)c->c_ci.p,
                                     c->c_v.p);
    int32_t kept = 0;
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_drop_zeros(s, (int32_t)out_dtype, A->rows, (const int32_t *)c->c_rp.p,
                                  nnz, (const int32_t *)c->c_ci.p, c->c_v.p, c->dz.p, dz_b,
                                  (int32_t *)c->o_rp.p, (int32_t *)c->o_ci.p, c->o_v.p, &kept);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_status(c->plan, s);
    if (st != RVSP_SUCCESS)
        goto done;
    {
        const size_t kn = (size_t)(kept > 0 ? kept : 1);
        h_rp = (int32_t *)rvsp_malloc(rp_b);
        h_ci = (int32_t *)rvsp_malloc(kn * sizeof(int32_t));
        h_v = rvsp_malloc(kn * out_sz);
        if (!h_rp || !h_ci || !h_v) {
            st = RVSP_ERROR_ALLOCATION_FAILED;
            goto done;
        }
        cudaError_t e = cudaMemcpyAsync(h_rp, c->o_rp.p, rp_b, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && kept > 0)
            e = cudaMemcpyAsync(h_ci, c->o_ci.p, (size_t)kept * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && kept > 0)
            e = cudaMemcpyAsync(h_v, c->o_v.p, (size_t)kept * out_sz, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            st = rvsp_map_cuda(e);
            goto done;
        }
        C->nnz = kept;
    }
out:
    if (A->rows == 0)
        C->nnz = 0;
    C->rows = A->rows;
    C->cols = B->cols;
    C->row_ptr = h_rp;
    C->col_idx = h_ci;
    C->values = h_v;
    C->dtype = out_dtype;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = 1;
    return RVSP_SUCCESS;
done:
    free(h_rp);
    free(h_ci);
    free(h_v);
    return st;
}
