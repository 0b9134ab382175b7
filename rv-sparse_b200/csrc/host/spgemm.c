/*
 * One-shot SpGEMM dispatch, the CUDA form of src/core/spgemm.c:26-211 of
 * merledu/rv-sparse.
 *
 * rvsp_spgemm_csr keeps the reference contract: NULL operands are rejected,
 * NULL options select this library's default backend (CUDA, FP32 -> FP32),
 * non-FP32 operands give UNSUPPORTED_DTYPE, A.cols != B.rows gives
 * INVALID_ARGUMENT, non-canonical CSR gives INVALID_CSR, C's arrays are
 * malloc'd by the library with owns_data = 1, and on failure C is nulled.
 * CPU backends are not provided: RVSP_BACKEND_SCALAR, _SCALAR_UNROLL4 and
 * _RVV_INTRINSICS report UNSUPPORTED_BACKEND.  RVSP_BACKEND_CUDA with
 * {FP64, FP64} or {INT8, INT32} runs the legacy kernels' products on the GPU
 * (typed.c, the reference's spgemm.c:179-193).
 *
 * Each host thread keeps one cached device context (plan, stream, device
 * buffers) for one-shot calls, created on first use and released when the
 * thread exits, so repeated one-shot products do not pay cudaMalloc/cudaFree.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "rvsp_internal.h"

typedef struct {
    rvsp_cuda_plan_t plan;
    cudaStream_t stream;
    rvsp_dev_csr_t dA, dB;
    rvsp_dbuf_t c_row_ptr, c_col, c_val, ws;
} oneshot_ctx_t;

static pthread_key_t g_ctx_key;
static pthread_once_t g_ctx_once = PTHREAD_ONCE_INIT;

static void ctx_free(void *p)
{
    oneshot_ctx_t *c = (oneshot_ctx_t *)p;
    if (!c)
        return;
    if (c->stream)
        cudaStreamSynchronize(c->stream);
    rvsp_cuda_plan_destroy(c->plan);
    rvsp_dev_csr_release(&c->dA);
    rvsp_dev_csr_release(&c->dB);
    rvsp_dbuf_release(&c->c_row_ptr);
    rvsp_dbuf_release(&c->c_col);
    rvsp_dbuf_release(&c->c_val);
    rvsp_dbuf_release(&c->ws);
    if (c->stream)
        cudaStreamDestroy(c->stream);
    free(c);
}

static void ctx_key_init(void)
{
    pthread_key_create(&g_ctx_key, ctx_free);
}

static rvsp_status_t get_ctx(oneshot_ctx_t **out)
{
    pthread_once(&g_ctx_once, ctx_key_init);
    oneshot_ctx_t *c = (oneshot_ctx_t *)pthread_getspecific(g_ctx_key);
    if (!c) {
        c = (oneshot_ctx_t *)rvsp_calloc(1, sizeof(*c));
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
        pthread_setspecific(g_ctx_key, c);
    }
    *out = c;
    return RVSP_SUCCESS;
}

/* Reference order of checks for the one-shot FP32 path (spgemm.c:31-51 then
 * check_operand inside the descriptor, spgemm_descr.c:137-160). */
static rvsp_status_t precheck(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B)
{
    if (A->dtype != RVSP_DTYPE_FP32 || B->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return RVSP_SUCCESS;
}

static void null_c(rvsp_csr_matrix_t *C)
{
    C->row_ptr = NULL;
    C->col_idx = NULL;
    C->values = NULL;
    C->nnz = 0;
    C->owns_data = 0;
}

/* Runs check -> symbolic -> numeric on device operands and leaves C's device
 * arrays in the context buffers. */
static rvsp_status_t run_device(oneshot_ctx_t *c, const rvsp_csr_matrix_t *A,
                                const rvsp_csr_matrix_t *B, const int32_t *a_rp,
                                const int32_t *a_ci, const float *a_v,
                                int32_t a_entries, const int32_t *b_rp,
                                const int32_t *b_ci, const float *b_v,
                                int32_t b_entries, int b_is_a, int64_t *c_nnz)
{
    rvsp_status_t st = rvsp_device_check(c->plan, c->stream, A->rows, A->cols, a_rp,
                                         a_ci, a_entries, RVSP_REJECT_ALL);
    if (st == RVSP_SUCCESS && !b_is_a)
        st = rvsp_device_check(c->plan, c->stream, B->rows, B->cols, b_rp, b_ci,
                               b_entries, RVSP_REJECT_ALL);
    if (st != RVSP_SUCCESS)
        return st;
    /* The descriptor-path operand checks come after the canonical check. */
    st = rvsp_check_operand(A);
    if (st == RVSP_SUCCESS)
        st = rvsp_check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_dbuf_reserve(&c->c_row_ptr, ((size_t)A->rows + 1) * sizeof(int32_t));
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_cuda_symbolic(c->plan, c->stream, A->rows, B->rows, B->cols, a_rp, a_ci,
                            b_rp, b_ci, (int32_t *)c->c_row_ptr.p, c_nnz);
    if (st != RVSP_SUCCESS)
        return st;
    const size_t n = (size_t)(*c_nnz > 0 ? *c_nnz : 1);
    st = rvsp_dbuf_reserve(&c->c_col, n * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&c->c_val, n * sizeof(float));
    const size_t ws = rvsp_cuda_numeric_workspace_bytes(c->plan);
    if (st == RVSP_SUCCESS && ws > 0)
        st = rvsp_dbuf_reserve(&c->ws, ws);
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_cuda_numeric(c->plan, c->stream, a_rp, a_ci, a_v, b_rp, b_ci, b_v,
                           (const int32_t *)c->c_row_ptr.p, (int32_t *)c->c_col.p,
                           (float *)c->c_val.p, 1, ws > 0 ? c->ws.p : NULL, ws);
    if (st != RVSP_SUCCESS)
        return st;
    return rvsp_cuda_plan_status(c->plan, c->stream);
}

static rvsp_status_t oneshot_host(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                                  rvsp_csr_matrix_t *C)
{
    rvsp_status_t st = precheck(A, B);
    if (st != RVSP_SUCCESS)
        return st;
    if (rvsp_csr_precheck(A) != RVSP_CSR_OK || rvsp_csr_precheck(B) != RVSP_CSR_OK)
        return RVSP_ERROR_INVALID_CSR;
    if (A->rows == 0 || B->rows == 0 || A->cols == 0 || B->cols == 0 || !A->col_idx ||
        !B->col_idx) {
        /* The canonical check had no column left to read and passed; the
         * descriptor's operand checks decide, as in the reference. */
        st = rvsp_check_operand(A);
        if (st == RVSP_SUCCESS)
            st = rvsp_check_operand(B);
        return st != RVSP_SUCCESS ? st : RVSP_ERROR_INVALID_ARGUMENT;
    }

    oneshot_ctx_t *c = NULL;
    st = get_ctx(&c);
    if (st != RVSP_SUCCESS)
        return st;
    cudaStream_t s = c->stream;
    const int b_is_a = A->row_ptr == B->row_ptr && A->col_idx == B->col_idx &&
                       A->rows == B->rows && A->cols == B->cols;
    const int bv_is_av = b_is_a && A->values == B->values;

    st = rvsp_dev_csr_upload_structure(&c->dA, A, s);
    if (st == RVSP_SUCCESS && !b_is_a)
        st = rvsp_dev_csr_upload_structure(&c->dB, B, s);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->values)
        st = rvsp_dev_csr_upload_values(&c->dA, A, s);
    if (st == RVSP_SUCCESS && B->values && !bv_is_av) {
        if (b_is_a)
            c->dB.entries = c->dA.entries;
        st = rvsp_dev_csr_upload_values(&c->dB, B, s);
    }
    if (st != RVSP_SUCCESS)
        return st;
    const rvsp_dev_csr_t *bs = b_is_a ? &c->dA : &c->dB;
    int64_t c_nnz = 0;
    st = run_device(c, A, B, (const int32_t *)c->dA.row_ptr.p,
                    (const int32_t *)c->dA.col_idx.p, (const float *)c->dA.values.p,
                    c->dA.entries, (const int32_t *)bs->row_ptr.p,
                    (const int32_t *)bs->col_idx.p,
                    (const float *)(bv_is_av ? c->dA.values.p : c->dB.values.p),
                    bs->entries, b_is_a, &c_nnz);
    if (st != RVSP_SUCCESS)
        return st;

    const size_t alloc = (size_t)(c_nnz > 0 ? c_nnz : 1);
    int32_t *rp = (int32_t *)rvsp_malloc(((size_t)A->rows + 1) * sizeof(int32_t));
    int32_t *ci = (int32_t *)rvsp_malloc(alloc * sizeof(int32_t));
    float *cv = (float *)rvsp_malloc(alloc * sizeof(float));
    if (!rp || !ci || !cv) {
        free(rp);
        free(ci);
        free(cv);
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    cudaError_t e = cudaMemcpyAsync(rp, c->c_row_ptr.p,
                                    ((size_t)A->rows + 1) * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && c_nnz > 0)
        e = cudaMemcpyAsync(ci, c->c_col.p, (size_t)c_nnz * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && c_nnz > 0)
        e = cudaMemcpyAsync(cv, c->c_val.p, (size_t)c_nnz * sizeof(float),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free(rp);
        free(ci);
        free(cv);
        return rvsp_map_cuda(e);
    }
    C->rows = A->rows;
    C->cols = B->cols;
    C->nnz = (int32_t)c_nnz;
    C->row_ptr = rp;
    C->col_idx = ci;
    C->values = cv;
    C->dtype = RVSP_DTYPE_FP32;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = 1;
    return RVSP_SUCCESS;
}

static rvsp_status_t resolve_options(const rvsp_spgemm_options_t *options, int *is_cuda)
{
    rvsp_backend_t backend = RVSP_BACKEND_CUDA;
    rvsp_dtype_t in = RVSP_DTYPE_FP32, out = RVSP_DTYPE_FP32;
    if (options) {
        backend = options->backend;
        in = options->input_dtype;
        out = options->output_dtype;
    }
    *is_cuda = backend == RVSP_BACKEND_CUDA && in == RVSP_DTYPE_FP32 &&
               out == RVSP_DTYPE_FP32;
    return *is_cuda ? RVSP_SUCCESS : RVSP_ERROR_UNSUPPORTED_BACKEND;
}

rvsp_status_t rvsp_spgemm_csr(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                              rvsp_csr_matrix_t *C,
                              const rvsp_spgemm_options_t *options)
{
    if (!A || !B || !C)
        return RVSP_ERROR_NULL_POINTER;
    /* FP64 and INT8 -> INT32: the legacy kernels' products (typed.c) */
    if (options && options->backend == RVSP_BACKEND_CUDA &&
        ((options->input_dtype == RVSP_DTYPE_FP64 && options->output_dtype == RVSP_DTYPE_FP64) ||
         (options->input_dtype == RVSP_DTYPE_INT8 && options->output_dtype == RVSP_DTYPE_INT32))) {
        rvsp_status_t ts = rvsp_typed_oneshot(A, B, C, options->input_dtype);
        if (ts != RVSP_SUCCESS)
            null_c(C);
        return ts;
    }
    int is_cuda = 0;
    rvsp_status_t st = resolve_options(options, &is_cuda);
    if (st != RVSP_SUCCESS)
        return st;
    st = oneshot_host(A, B, C);
    if (st != RVSP_SUCCESS)
        null_c(C);
    return st;
}

rvsp_status_t rvsp_spgemm_csr_device(const rvsp_csr_matrix_t *A,
                                     const rvsp_csr_matrix_t *B, rvsp_csr_matrix_t *C,
                                     const rvsp_spgemm_options_t *options)
{
    if (!A || !B || !C)
        return RVSP_ERROR_NULL_POINTER;
    int is_cuda = 0;
    rvsp_status_t st = resolve_options(options, &is_cuda);
    if (st != RVSP_SUCCESS)
        return st;
    st = precheck(A, B);
    if (st == RVSP_SUCCESS && (!A->row_ptr || !B->row_ptr))
        st = RVSP_ERROR_INVALID_CSR;
    if (st == RVSP_SUCCESS && (A->rows <= 0 || B->rows <= 0 || A->cols <= 0 ||
                               B->cols <= 0 || A->nnz < 0 || B->nnz < 0))
        st = RVSP_ERROR_INVALID_ARGUMENT;
    oneshot_ctx_t *c = NULL;
    if (st == RVSP_SUCCESS)
        st = get_ctx(&c);
    int64_t c_nnz = 0;
    if (st == RVSP_SUCCESS) {
        const int b_is_a = A->row_ptr == B->row_ptr && A->col_idx == B->col_idx;
        st = run_device(c, A, B, A->row_ptr, A->col_idx, (const float *)A->values,
                        A->nnz, B->row_ptr, B->col_idx, (const float *)B->values,
                        B->nnz, b_is_a, &c_nnz);
    }
    if (st != RVSP_SUCCESS) {
        null_c(C);
        return st;
    }
    /* Hand the context's C buffers to the caller; the context grows new ones
     * on its next call. */
    C->rows = A->rows;
    C->cols = B->cols;
    C->nnz = (int32_t)c_nnz;
    C->row_ptr = (int32_t *)c->c_row_ptr.p;
    C->col_idx = (int32_t *)c->c_col.p;
    C->values = c->c_val.p;
    C->dtype = RVSP_DTYPE_FP32;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = 2;
    c->c_row_ptr.p = NULL;
    c->c_row_ptr.cap = 0;
    c->c_col.p = NULL;
    c->c_col.cap = 0;
    c->c_val.p = NULL;
    c->c_val.cap = 0;
    return RVSP_SUCCESS;
}
