/*
 * Batches of independent products (new API; no reference counterpart: the
 * reference computes one product per rvsp_spgemm_csr or descriptor call,
 * spgemm.c:135-210 and spgemm_descr.c:66-380).
 *
 * Layout.  Products are taken in order into groups whose op counts sum to at
 * most group_ops (INT32_MAX by default, which keeps every group's nnz(C) in
 * int32).  A group is one operand pair on the device: A_g stacks the A_i
 * with column indices offset by the first row of B_i inside B_g, B_g stacks
 * the B_i with their own columns (rvsp_cuda_batch_pack).  Row r of A_g * B_g
 * is the matching row of its C_i with the same terms in the same order, so
 * one plan per group (rvsp_cuda_symbolic / rvsp_cuda_numeric: one launch per
 * row class over the rows of every product in the group) gives results
 * bit-identical to computing each product alone.
 *
 * Host memory space copies every operand once into one device arena; device
 * memory space reads the caller's arrays.  Either way the packs are the
 * batch's own, so each compute first refreshes their values from the
 * operands (a copy kernel, after uploads in host memory space).
 *
 * Repeats.  The first compute fills columns and values.  Every later compute
 * is numeric-only: the first such call records [value refresh + numeric pass
 * of every group] into a CUDA graph (relaxed capture mode) and the following
 * ones replay it.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rvsp_internal.h"

typedef struct {
    int32_t first, count;           /* products [first, first + count) */
    int32_t a_rows, b_rows, b_cols; /* of the packed pair */
    int32_t a_nnz, b_nnz;
    int64_t ops;
    rvsp_dbuf_t off;                /* rvsp_cuda_batch_offset_t[count] */
    rvsp_dbuf_t a_rp, a_ci, a_v, b_rp, b_ci, b_v;
    rvsp_cuda_plan_t plan;
    int32_t c_nnz;
    rvsp_dbuf_t c_rp, c_ci, c_v, ws;
    size_t ws_bytes;
} batch_group_t;

struct rvsp_spgemm_batch {
    rvsp_memory_space_t mem;
    cudaStream_t stream, own_stream;
    int user_stream;
    int autotune;
    int32_t merge_policy;
    int32_t persist_rows, persist_blocks; /* persistent numeric-only pass */
    float tuned_ms[8];                    /* autotuner timings (see get_tuning) */
    int32_t n_tuned;
    int64_t group_ops;

    int32_t count, cap;
    rvsp_csr_matrix_t *A, *B;       /* the caller's structs */

    int estimated, filled;
    rvsp_cuda_batch_item_t *h_items;
    rvsp_dbuf_t d_items, d_ops, d_err;
    int64_t *h_ops;
    int64_t total_ops;

    /* host memory space: one arena with every operand's arrays */
    rvsp_dbuf_t raw_i32, raw_f32;
    int64_t *raw_val_off;           /* per product: a values, b values (floats) */

    int32_t ngroups;
    batch_group_t *groups;
    int32_t *group_of;              /* per product */

    rvsp_dbuf_t crp_all, d_crp_off, d_base, d_nnz;
    int64_t *crp_off;               /* per product, into crp_all */
    int32_t *base, *nnz;            /* per product, into its group's C */
    int64_t total_nnz;

    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

static void drop_graph(rvsp_spgemm_batch_t b)
{
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    b->exec = NULL;
    b->graph = NULL;
}

static void release_group(batch_group_t *g)
{
    rvsp_dbuf_release(&g->off);
    rvsp_dbuf_release(&g->a_rp);
    rvsp_dbuf_release(&g->a_ci);
    rvsp_dbuf_release(&g->a_v);
    rvsp_dbuf_release(&g->b_rp);
    rvsp_dbuf_release(&g->b_ci);
    rvsp_dbuf_release(&g->b_v);
    rvsp_dbuf_release(&g->c_rp);
    rvsp_dbuf_release(&g->c_ci);
    rvsp_dbuf_release(&g->c_v);
    rvsp_dbuf_release(&g->ws);
    if (g->plan)
        rvsp_cuda_plan_destroy(g->plan);
    memset(g, 0, sizeof(*g));
}

/* Discards the analysis (groups, views, graph). */
static void reset_analysis(rvsp_spgemm_batch_t b)
{
    drop_graph(b);
    for (int32_t i = 0; i < b->ngroups; i++)
        release_group(&b->groups[i]);
    free(b->groups);
    b->groups = NULL;
    b->ngroups = 0;
    free(b->h_items);
    free(b->h_ops);
    free(b->raw_val_off);
    free(b->group_of);
    free(b->crp_off);
    free(b->base);
    free(b->nnz);
    b->h_items = NULL;
    b->h_ops = NULL;
    b->raw_val_off = NULL;
    b->group_of = NULL;
    b->crp_off = NULL;
    b->base = NULL;
    b->nnz = NULL;
    b->estimated = 0;
    b->filled = 0;
    b->total_nnz = 0;
    b->total_ops = 0;
}

rvsp_status_t rvsp_spgemm_batch_create(rvsp_spgemm_batch_t *batch)
{
    if (batch == NULL)
        return RVSP_ERROR_NULL_POINTER;
    *batch = NULL;
    struct rvsp_spgemm_batch *b = (struct rvsp_spgemm_batch *)rvsp_calloc(1, sizeof(*b));
    if (b == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    b->mem = RVSP_MEM_HOST;
    b->group_ops = INT32_MAX;
    *batch = b;
    return RVSP_SUCCESS;
}

void rvsp_spgemm_batch_destroy(rvsp_spgemm_batch_t b)
{
    if (b == NULL)
        return;
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    reset_analysis(b);
    rvsp_dbuf_release(&b->d_items);
    rvsp_dbuf_release(&b->d_ops);
    rvsp_dbuf_release(&b->d_err);
    rvsp_dbuf_release(&b->raw_i32);
    rvsp_dbuf_release(&b->raw_f32);
    rvsp_dbuf_release(&b->crp_all);
    rvsp_dbuf_release(&b->d_crp_off);
    rvsp_dbuf_release(&b->d_base);
    rvsp_dbuf_release(&b->d_nnz);
    if (b->own_stream)
        cudaStreamDestroy(b->own_stream);
    free(b->A);
    free(b->B);
    free(b);
}

rvsp_status_t rvsp_spgemm_batch_set_memory_space(rvsp_spgemm_batch_t b,
                                                 rvsp_memory_space_t space)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (space != RVSP_MEM_HOST && space != RVSP_MEM_DEVICE)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (b->count > 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    b->mem = space;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_set_stream(rvsp_spgemm_batch_t b, void *stream)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    drop_graph(b); /* a graph is replayed on the stream it was made for */
    b->user_stream = stream != NULL;
    b->stream = stream != NULL ? (cudaStream_t)stream : b->own_stream;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_set_autotune(rvsp_spgemm_batch_t b, int enable)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    b->autotune = enable != 0;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_set_persistent(rvsp_spgemm_batch_t b, int32_t merge_rows,
                                               int32_t blocks_per_sm)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (merge_rows < 0 || merge_rows > 256 || merge_rows % 32 != 0 || blocks_per_sm < 1 ||
        blocks_per_sm > 4 || b->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    b->persist_rows = merge_rows;
    b->persist_blocks = blocks_per_sm;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_get_tuning(rvsp_spgemm_batch_t b, int32_t *merge_policy_out,
                                           int32_t *merge_rows_out, int32_t *blocks_out,
                                           float *shape_ms_out, int32_t *n_shapes_out)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (merge_policy_out)
        *merge_policy_out = b->merge_policy;
    if (merge_rows_out)
        *merge_rows_out = b->persist_rows;
    if (blocks_out)
        *blocks_out = b->persist_blocks > 0 ? b->persist_blocks : 2;
    if (shape_ms_out)
        for (int32_t i = 0; i < b->n_tuned; i++)
            shape_ms_out[i] = b->tuned_ms[i];
    if (n_shapes_out)
        *n_shapes_out = b->n_tuned;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_set_merge_policy(rvsp_spgemm_batch_t b, int32_t policy)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (policy < 0 || policy > 2 || b->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    b->merge_policy = policy;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_set_group_ops(rvsp_spgemm_batch_t b, int64_t max_ops)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (max_ops <= 0 || max_ops > INT32_MAX || b->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    b->group_ops = max_ops;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_add(rvsp_spgemm_batch_t b, const rvsp_csr_matrix_t *A,
                                    const rvsp_csr_matrix_t *B, int32_t *index_out)
{
    if (b == NULL || A == NULL || B == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (b->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    rvsp_status_t st = rvsp_check_operand(A);
    if (st == RVSP_SUCCESS)
        st = rvsp_check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (b->count == b->cap) {
        const int32_t cap = b->cap ? 2 * b->cap : 64;
        rvsp_csr_matrix_t *na = (rvsp_csr_matrix_t *)rvsp_realloc(b->A, (size_t)cap * sizeof(*na));
        if (na == NULL)
            return RVSP_ERROR_ALLOCATION_FAILED;
        b->A = na;
        rvsp_csr_matrix_t *nb = (rvsp_csr_matrix_t *)rvsp_realloc(b->B, (size_t)cap * sizeof(*nb));
        if (nb == NULL)
            return RVSP_ERROR_ALLOCATION_FAILED;
        b->B = nb;
        b->cap = cap;
    }
    b->A[b->count] = *A;
    b->B[b->count] = *B;
    if (index_out)
        *index_out = b->count;
    b->count++;
    return RVSP_SUCCESS;
}

static rvsp_status_t ensure_stream(rvsp_spgemm_batch_t b)
{
    if (!b->own_stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
    }
    if (!b->user_stream)
        b->stream = b->own_stream;
    return RVSP_SUCCESS;
}

static rvsp_status_t cuda_ok(cudaError_t e)
{
    return e == cudaSuccess ? RVSP_SUCCESS : rvsp_map_cuda(e);
}

/* Host memory space: canonical check of every operand on the host, then one
 * device arena holding all of their arrays; items point into it. */
static rvsp_status_t stage_host_operands(rvsp_spgemm_batch_t b)
{
    int64_t n_i32 = 0, n_f32 = 0;
    for (int32_t i = 0; i < b->count; i++) {
        const rvsp_csr_matrix_t *M[2] = {&b->A[i], &b->B[i]};
        for (int k = 0; k < 2; k++) {
            int32_t bad = -1;
            if (rvsp_csr_check(M[k]->rows, M[k]->cols, M[k]->row_ptr, M[k]->col_idx, &bad) !=
                RVSP_CSR_OK)
                return RVSP_ERROR_INVALID_CSR;
            const int64_t entries = M[k]->row_ptr[M[k]->rows];
            n_i32 += (int64_t)M[k]->rows + 1 + entries;
            n_f32 += entries;
        }
    }
    rvsp_status_t st = rvsp_dbuf_reserve(&b->raw_i32, (size_t)n_i32 * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->raw_f32, (size_t)(n_f32 > 0 ? n_f32 : 1) * sizeof(float));
    if (st != RVSP_SUCCESS)
        return st;
    b->raw_val_off = (int64_t *)rvsp_malloc((size_t)(uint32_t)b->count * 2 * sizeof(int64_t));
    if (b->raw_val_off == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    int32_t *i32 = (int32_t *)b->raw_i32.p;
    float *f32 = (float *)b->raw_f32.p;
    int64_t oi = 0, of = 0;
    cudaError_t e = cudaSuccess;
    for (int32_t i = 0; i < b->count && e == cudaSuccess; i++) {
        rvsp_cuda_batch_item_t *it = &b->h_items[i];
        const rvsp_csr_matrix_t *M[2] = {&b->A[i], &b->B[i]};
        for (int k = 0; k < 2 && e == cudaSuccess; k++) {
            const int32_t rows = M[k]->rows, entries = M[k]->row_ptr[rows];
            int32_t *rp = i32 + oi, *ci = rp + rows + 1;
            float *v = f32 + of;
            e = cudaMemcpyAsync(rp, M[k]->row_ptr, ((size_t)rows + 1) * sizeof(int32_t),
                                cudaMemcpyHostToDevice, b->stream);
            if (e == cudaSuccess && entries > 0)
                e = cudaMemcpyAsync(ci, M[k]->col_idx, (size_t)entries * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, b->stream);
            b->raw_val_off[2 * i + k] = of;
            if (k == 0) {
                it->a_row_ptr = rp;
                it->a_col_idx = ci;
                it->a_values = v;
                it->a_nnz = entries;
            } else {
                it->b_row_ptr = rp;
                it->b_col_idx = ci;
                it->b_values = v;
                it->b_nnz = entries;
            }
            oi += (int64_t)rows + 1 + entries;
            of += entries;
        }
    }
    return cuda_ok(e);
}

/* Host memory space: uploads every operand's values into the arena. */
static rvsp_status_t upload_host_values(rvsp_spgemm_batch_t b)
{
    float *f32 = (float *)b->raw_f32.p;
    cudaError_t e = cudaSuccess;
    for (int32_t i = 0; i < b->count && e == cudaSuccess; i++) {
        const rvsp_cuda_batch_item_t *it = &b->h_items[i];
        if (it->a_nnz > 0)
            e = cudaMemcpyAsync(f32 + b->raw_val_off[2 * i], b->A[i].values,
                                (size_t)it->a_nnz * sizeof(float), cudaMemcpyHostToDevice,
                                b->stream);
        if (e == cudaSuccess && it->b_nnz > 0)
            e = cudaMemcpyAsync(f32 + b->raw_val_off[2 * i + 1], b->B[i].values,
                                (size_t)it->b_nnz * sizeof(float), cudaMemcpyHostToDevice,
                                b->stream);
    }
    return cuda_ok(e);
}

/* Reads the device error word (after a sync) and clears it. */
static rvsp_status_t take_error(rvsp_spgemm_batch_t b)
{
    int32_t err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, b->d_err.p, sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(b->d_err.p, 0, sizeof(int32_t), b->stream);
    if (e != cudaSuccess)
        return rvsp_map_cuda(e);
    return err ? RVSP_ERROR_INVALID_CSR : RVSP_SUCCESS;
}

/* Forms the groups: products in order, each group's op count <= group_ops
 * and its packed entry and row counts within int32. */
static rvsp_status_t form_groups(rvsp_spgemm_batch_t b)
{
    const size_t n = (size_t)(uint32_t)b->count;
    b->groups = (batch_group_t *)rvsp_calloc(n, sizeof(batch_group_t));
    b->group_of = (int32_t *)rvsp_malloc(n * sizeof(int32_t));
    if (b->groups == NULL || b->group_of == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    int32_t ng = 0;
    batch_group_t *g = NULL;
    for (int32_t i = 0; i < b->count; i++) {
        const rvsp_cuda_batch_item_t *it = &b->h_items[i];
        int fits = g != NULL;
        if (fits) {
            fits = g->ops + b->h_ops[i] <= b->group_ops &&
                   (int64_t)g->a_rows + it->a_rows < INT32_MAX &&
                   (int64_t)g->b_rows + it->b_rows < INT32_MAX &&
                   (int64_t)g->a_nnz + it->a_nnz < INT32_MAX &&
                   (int64_t)g->b_nnz + it->b_nnz < INT32_MAX;
        }
        if (!fits) {
            g = &b->groups[ng++];
            g->first = i;
        }
        g->count++;
        g->ops += b->h_ops[i];
        g->a_rows += it->a_rows;
        g->b_rows += it->b_rows;
        g->a_nnz += it->a_nnz;
        g->b_nnz += it->b_nnz;
        if (it->b_cols > g->b_cols)
            g->b_cols = it->b_cols;
        b->group_of[i] = ng - 1;
    }
    b->ngroups = ng;
    return RVSP_SUCCESS;
}

/* Packs group g (structure and values) and checks the packed operands. */
static rvsp_status_t pack_group(rvsp_spgemm_batch_t b, batch_group_t *g)
{
    rvsp_cuda_batch_offset_t *off =
        (rvsp_cuda_batch_offset_t *)rvsp_malloc((size_t)(uint32_t)g->count * sizeof(*off));
    if (off == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    int32_t ar = 0, an = 0, br = 0, bn = 0;
    for (int32_t j = 0; j < g->count; j++) {
        const rvsp_cuda_batch_item_t *it = &b->h_items[g->first + j];
        off[j].a_row = ar;
        off[j].a_nnz = an;
        off[j].b_row = br;
        off[j].b_nnz = bn;
        ar += it->a_rows;
        an += it->a_nnz;
        br += it->b_rows;
        bn += it->b_nnz;
    }
    rvsp_status_t st = rvsp_dbuf_reserve(&g->off, (size_t)g->count * sizeof(*off));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(g->off.p, off, (size_t)g->count * sizeof(*off),
                                     cudaMemcpyHostToDevice, b->stream));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaStreamSynchronize(b->stream)); /* off is freed below */
    free(off);
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->a_rp, ((size_t)g->a_rows + 1) * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->a_ci, (size_t)g->a_nnz * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->a_v, (size_t)g->a_nnz * sizeof(float));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->b_rp, ((size_t)g->b_rows + 1) * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->b_ci, (size_t)g->b_nnz * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->b_v, (size_t)g->b_nnz * sizeof(float));
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_create(&g->plan);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_plan_set_merge_policy(g->plan, b->merge_policy);
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_batch_pack(b->stream, (const rvsp_cuda_batch_item_t *)b->d_items.p +
                                                 g->first,
                                  (const rvsp_cuda_batch_offset_t *)g->off.p, g->count, 1,
                                  (int32_t *)g->a_rp.p, (int32_t *)g->a_ci.p,
                                  (float *)g->a_v.p, (int32_t *)g->b_rp.p,
                                  (int32_t *)g->b_ci.p, (float *)g->b_v.p,
                                  (int32_t *)b->d_err.p);
    if (st == RVSP_SUCCESS)
        st = take_error(b);
    /* Sorted, duplicate-free rows and monotone row pointers of the packs are
     * those of the operands; column ranges were checked per product above. */
    if (st == RVSP_SUCCESS)
        st = rvsp_device_check(g->plan, b->stream, g->a_rows, g->b_rows,
                               (const int32_t *)g->a_rp.p, (const int32_t *)g->a_ci.p,
                               g->a_nnz, RVSP_REJECT_ALL);
    if (st == RVSP_SUCCESS)
        st = rvsp_device_check(g->plan, b->stream, g->b_rows, g->b_cols,
                               (const int32_t *)g->b_rp.p, (const int32_t *)g->b_ci.p,
                               g->b_nnz, RVSP_REJECT_ALL);
    return st;
}

/* Structure of group g: C_g.row_ptr, nnz, C arrays and workspace. */
static rvsp_status_t analyse_group(rvsp_spgemm_batch_t b, batch_group_t *g)
{
    rvsp_status_t st =
        rvsp_dbuf_reserve(&g->c_rp, ((size_t)g->a_rows + 1) * sizeof(int32_t));
    int64_t total = 0;
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_symbolic(g->plan, b->stream, g->a_rows, g->b_rows, g->b_cols,
                                (const int32_t *)g->a_rp.p, (const int32_t *)g->a_ci.p,
                                (const int32_t *)g->b_rp.p, (const int32_t *)g->b_ci.p,
                                (int32_t *)g->c_rp.p, &total);
    if (st != RVSP_SUCCESS)
        return st;
    g->c_nnz = (int32_t)total;
    st = rvsp_dbuf_reserve(&g->c_ci, (size_t)g->c_nnz * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->c_v, (size_t)g->c_nnz * sizeof(float));
    const size_t need = rvsp_cuda_numeric_workspace_bytes(g->plan);
    g->ws_bytes = need > 256 ? need : 256;
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&g->ws, g->ws_bytes);
    return st;
}

/* Numeric pass of every group; fill = columns too.  Values are refreshed
 * from the operands first. */
static rvsp_status_t run_groups(rvsp_spgemm_batch_t b, int fill)
{
    rvsp_status_t st = RVSP_SUCCESS;
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++) {
        batch_group_t *g = &b->groups[k];
        st = rvsp_cuda_batch_pack(b->stream,
                                  (const rvsp_cuda_batch_item_t *)b->d_items.p + g->first,
                                  (const rvsp_cuda_batch_offset_t *)g->off.p, g->count, 0,
                                  NULL, NULL, (float *)g->a_v.p, NULL, NULL,
                                  (float *)g->b_v.p, (int32_t *)b->d_err.p);
        if (st == RVSP_SUCCESS)
            st = rvsp_cuda_numeric(g->plan, b->stream, (const int32_t *)g->a_rp.p,
                                   (const int32_t *)g->a_ci.p, (const float *)g->a_v.p,
                                   (const int32_t *)g->b_rp.p, (const int32_t *)g->b_ci.p,
                                   (const float *)g->b_v.p, (const int32_t *)g->c_rp.p,
                                   (int32_t *)g->c_ci.p, (float *)g->c_v.p, fill, g->ws.p,
                                   g->ws_bytes);
    }
    return st;
}

/* Milliseconds of one numeric-only pass of every group (events, best of 2
 * after a warm pass). */
static rvsp_status_t time_numeric(rvsp_spgemm_batch_t b, float *ms_out)
{
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess)
        return RVSP_ERROR_DEVICE;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return RVSP_ERROR_DEVICE;
    }
    rvsp_status_t st = run_groups(b, 0);
    float best = 0.0f;
    for (int rep = 0; rep < 2 && st == RVSP_SUCCESS; rep++) {
        cudaEventRecord(e0, b->stream);
        st = run_groups(b, 0);
        cudaEventRecord(e1, b->stream);
        if (st == RVSP_SUCCESS)
            st = cuda_ok(cudaEventSynchronize(e1));
        float ms = 0.0f;
        if (st == RVSP_SUCCESS)
            cudaEventElapsedTime(&ms, e0, e1);
        if (rep == 0 || ms < best)
            best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_out = best;
    return st;
}

static rvsp_status_t set_persistent_all(rvsp_spgemm_batch_t b)
{
    rvsp_status_t st = RVSP_SUCCESS;
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++)
        st = rvsp_cuda_plan_set_persistent(b->groups[k].plan, b->persist_rows,
                                           b->persist_blocks > 0 ? b->persist_blocks : 2);
    return st;
}

static rvsp_status_t analyse_all(rvsp_spgemm_batch_t b)
{
    rvsp_status_t st = RVSP_SUCCESS;
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++) {
        st = rvsp_cuda_plan_set_merge_policy(b->groups[k].plan, b->merge_policy);
        if (st == RVSP_SUCCESS)
            st = analyse_group(b, &b->groups[k]);
    }
    if (st == RVSP_SUCCESS)
        st = set_persistent_all(b);
    return st;
}

/* Builds every group's reuse map for the structure of the last fill. */
static rvsp_status_t prepare_reuse_all(rvsp_spgemm_batch_t b)
{
    rvsp_status_t st = RVSP_SUCCESS;
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++) {
        const batch_group_t *g = &b->groups[k];
        st = rvsp_cuda_plan_prepare_reuse(g->plan, b->stream, (const int32_t *)g->a_rp.p,
                                          (const int32_t *)g->a_ci.p,
                                          (const int32_t *)g->b_rp.p,
                                          (const int32_t *)g->b_ci.p,
                                          (const int32_t *)g->c_rp.p,
                                          (const int32_t *)g->c_ci.p, NULL);
    }
    return st;
}

/* The numeric-only shapes the autotuner times: one launch per row class,
 * then the persistent pass with merge rows per bin x blocks per SM. */
static const int32_t kTuneShapes[][2] = {{0, 2}, {128, 2}, {256, 2}, {256, 1}, {64, 4}};
#define N_TUNE_SHAPES ((int32_t)(sizeof(kTuneShapes) / sizeof(kTuneShapes[0])))

/* Times each shape on the analysed batch (one fill, reuse maps built, then
 * numeric-only passes) and keeps the fastest. */
static rvsp_status_t autotune_shape(rvsp_spgemm_batch_t b)
{
    rvsp_status_t st = run_groups(b, 1);
    if (st == RVSP_SUCCESS)
        st = prepare_reuse_all(b);
    int32_t best = -1;
    float best_ms = 0.0f;
    b->n_tuned = 0;
    for (int32_t i = 0; i < N_TUNE_SHAPES && st == RVSP_SUCCESS; i++) {
        b->persist_rows = kTuneShapes[i][0];
        b->persist_blocks = kTuneShapes[i][1];
        st = set_persistent_all(b);
        float ms = 0.0f;
        if (st == RVSP_SUCCESS)
            st = time_numeric(b, &ms);
        if (st == RVSP_SUCCESS) {
            b->tuned_ms[b->n_tuned++] = ms;
            if (best < 0 || ms < best_ms) {
                best = i;
                best_ms = ms;
            }
        }
    }
    if (st != RVSP_SUCCESS)
        return st;
    b->persist_rows = kTuneShapes[best][0];
    b->persist_blocks = kTuneShapes[best][1];
    return set_persistent_all(b);
}

/* The autotuner: tries each merge policy on the batch (symbolic + one fill
 * + timed numeric-only passes) and keeps the fastest, analysed. */
static rvsp_status_t autotune_policy(rvsp_spgemm_batch_t b)
{
    float best_ms = 0.0f;
    int32_t best = -1;
    for (int32_t policy = 0; policy <= 2; policy++) {
        b->merge_policy = policy;
        rvsp_status_t st = analyse_all(b);
        if (st == RVSP_SUCCESS)
            st = run_groups(b, 1);
        float ms = 0.0f;
        if (st == RVSP_SUCCESS)
            st = time_numeric(b, &ms);
        if (st != RVSP_SUCCESS)
            return st;
        if (best < 0 || ms < best_ms) {
            best = policy;
            best_ms = ms;
        }
    }
    b->merge_policy = best;
    rvsp_status_t st = best == 2 ? RVSP_SUCCESS : analyse_all(b);
    if (st == RVSP_SUCCESS)
        st = autotune_shape(b);
    return st;
}

/* Per-product views of the groups' C: rebased row pointers, bases, nnz. */
static rvsp_status_t build_views(rvsp_spgemm_batch_t b)
{
    const size_t n = (size_t)(uint32_t)b->count;
    b->crp_off = (int64_t *)rvsp_malloc(n * sizeof(int64_t));
    b->base = (int32_t *)rvsp_malloc(n * sizeof(int32_t));
    b->nnz = (int32_t *)rvsp_malloc(n * sizeof(int32_t));
    if (b->crp_off == NULL || b->base == NULL || b->nnz == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    int64_t rows = 0;
    for (int32_t i = 0; i < b->count; i++) {
        b->crp_off[i] = rows;
        rows += (int64_t)b->h_items[i].a_rows + 1;
    }
    rvsp_status_t st = rvsp_dbuf_reserve(&b->crp_all, (size_t)rows * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->d_crp_off, n * sizeof(int64_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->d_base, n * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->d_nnz, n * sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(b->d_crp_off.p, b->crp_off, n * sizeof(int64_t),
                                     cudaMemcpyHostToDevice, b->stream));
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++) {
        const batch_group_t *g = &b->groups[k];
        st = rvsp_cuda_batch_views(b->stream,
                                   (const rvsp_cuda_batch_item_t *)b->d_items.p + g->first,
                                   (const rvsp_cuda_batch_offset_t *)g->off.p,
                                   (const int64_t *)b->d_crp_off.p + g->first, g->count,
                                   (const int32_t *)g->c_rp.p, (int32_t *)b->crp_all.p,
                                   (int32_t *)b->d_base.p + g->first,
                                   (int32_t *)b->d_nnz.p + g->first);
    }
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(b->base, b->d_base.p, n * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, b->stream));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(b->nnz, b->d_nnz.p, n * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, b->stream));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaStreamSynchronize(b->stream));
    b->total_nnz = 0;
    for (int32_t i = 0; i < b->count && st == RVSP_SUCCESS; i++)
        b->total_nnz += b->nnz[i];
    return st;
}

rvsp_status_t rvsp_spgemm_batch_work_estimation(rvsp_spgemm_batch_t b,
                                                int64_t *total_nnz_out)
{
    if (b == NULL || total_nnz_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (b->count == 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    reset_analysis(b);
    rvsp_status_t st = ensure_stream(b);
    if (st != RVSP_SUCCESS)
        return st;
    const size_t n = (size_t)(uint32_t)b->count;
    b->h_items = (rvsp_cuda_batch_item_t *)rvsp_calloc(n, sizeof(rvsp_cuda_batch_item_t));
    b->h_ops = (int64_t *)rvsp_calloc(n, sizeof(int64_t));
    if (b->h_items == NULL || b->h_ops == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    for (int32_t i = 0; i < b->count; i++) {
        rvsp_cuda_batch_item_t *it = &b->h_items[i];
        it->a_rows = b->A[i].rows;
        it->b_rows = b->B[i].rows;
        it->b_cols = b->B[i].cols;
        it->a_row_ptr = b->A[i].row_ptr;
        it->a_col_idx = b->A[i].col_idx;
        it->a_values = (const float *)b->A[i].values;
        it->b_row_ptr = b->B[i].row_ptr;
        it->b_col_idx = b->B[i].col_idx;
        it->b_values = (const float *)b->B[i].values;
    }
    st = rvsp_dbuf_reserve(&b->d_err, sizeof(int32_t));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemsetAsync(b->d_err.p, 0, sizeof(int32_t), b->stream));
    if (st == RVSP_SUCCESS && b->mem == RVSP_MEM_HOST)
        st = stage_host_operands(b);
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->d_items, n * sizeof(rvsp_cuda_batch_item_t));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(b->d_items.p, b->h_items, n * sizeof(rvsp_cuda_batch_item_t),
                                     cudaMemcpyHostToDevice, b->stream));
    if (st == RVSP_SUCCESS && b->mem == RVSP_MEM_DEVICE) {
        /* entry counts live in the caller's device row pointers */
        st = rvsp_cuda_batch_entries(b->stream, (rvsp_cuda_batch_item_t *)b->d_items.p,
                                     b->count);
        if (st == RVSP_SUCCESS)
            st = cuda_ok(cudaMemcpyAsync(b->h_items, b->d_items.p,
                                         n * sizeof(rvsp_cuda_batch_item_t),
                                         cudaMemcpyDeviceToHost, b->stream));
        if (st == RVSP_SUCCESS)
            st = cuda_ok(cudaStreamSynchronize(b->stream));
        for (int32_t i = 0; i < b->count && st == RVSP_SUCCESS; i++)
            if (b->h_items[i].a_nnz < 0 || b->h_items[i].b_nnz < 0)
                st = RVSP_ERROR_INVALID_CSR;
    }
    if (st == RVSP_SUCCESS)
        st = rvsp_dbuf_reserve(&b->d_ops, n * sizeof(int64_t));
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemsetAsync(b->d_ops.p, 0, n * sizeof(int64_t), b->stream));
    if (st == RVSP_SUCCESS)
        st = rvsp_cuda_batch_op_counts(b->stream, (const rvsp_cuda_batch_item_t *)b->d_items.p,
                                       b->count, (int64_t *)b->d_ops.p, (int32_t *)b->d_err.p);
    if (st == RVSP_SUCCESS)
        st = cuda_ok(cudaMemcpyAsync(b->h_ops, b->d_ops.p, n * sizeof(int64_t),
                                     cudaMemcpyDeviceToHost, b->stream));
    if (st == RVSP_SUCCESS)
        st = take_error(b);
    if (st != RVSP_SUCCESS)
        return st;
    b->total_ops = 0;
    for (int32_t i = 0; i < b->count; i++)
        b->total_ops += b->h_ops[i];

    st = form_groups(b);
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++)
        st = pack_group(b, &b->groups[k]);
    if (st == RVSP_SUCCESS)
        st = b->autotune ? autotune_policy(b) : analyse_all(b);
    if (st == RVSP_SUCCESS)
        st = build_views(b);
    if (st != RVSP_SUCCESS)
        return st;
    b->estimated = 1;
    *total_nnz_out = b->total_nnz;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_compute(rvsp_spgemm_batch_t b)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!b->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    rvsp_status_t st = RVSP_SUCCESS;
    if (b->mem == RVSP_MEM_HOST)
        st = upload_host_values(b);
    if (st != RVSP_SUCCESS)
        return st;
    if (!b->filled) {
        st = run_groups(b, 1);
        /* The repeats are captured, so build each group's reuse map now. */
        if (st == RVSP_SUCCESS)
            st = prepare_reuse_all(b);
        if (st == RVSP_SUCCESS)
            b->filled = 1;
        return st;
    }
    if (b->exec == NULL) {
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess)
            return rvsp_map_cuda(e);
        st = run_groups(b, 0);
        cudaGraph_t graph = NULL;
        e = cudaStreamEndCapture(b->stream, &graph);
        if (st == RVSP_SUCCESS && e != cudaSuccess)
            st = rvsp_map_cuda(e);
        if (st == RVSP_SUCCESS) {
            e = cudaGraphInstantiate(&b->exec, graph, 0);
            if (e != cudaSuccess) {
                b->exec = NULL;
                st = rvsp_map_cuda(e);
            }
        }
        if (st == RVSP_SUCCESS)
            b->graph = graph;
        else if (graph)
            cudaGraphDestroy(graph);
        if (st != RVSP_SUCCESS)
            return st;
    }
    return cuda_ok(cudaGraphLaunch(b->exec, b->stream));
}

rvsp_status_t rvsp_spgemm_batch_synchronize(rvsp_spgemm_batch_t b)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!b->stream)
        return RVSP_SUCCESS;
    rvsp_status_t st = cuda_ok(cudaStreamSynchronize(b->stream));
    for (int32_t k = 0; k < b->ngroups && st == RVSP_SUCCESS; k++)
        st = rvsp_cuda_plan_status(b->groups[k].plan, b->stream);
    return st;
}

rvsp_status_t rvsp_spgemm_batch_get_nnz(rvsp_spgemm_batch_t b, int32_t index,
                                        int32_t *nnz_out)
{
    if (b == NULL || nnz_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!b->estimated || index < 0 || index >= b->count)
        return RVSP_ERROR_INVALID_ARGUMENT;
    *nnz_out = b->nnz[index];
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_get_result(rvsp_spgemm_batch_t b, int32_t index,
                                           rvsp_csr_matrix_t *C_out)
{
    if (b == NULL || C_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!b->estimated || index < 0 || index >= b->count)
        return RVSP_ERROR_INVALID_ARGUMENT;
    const batch_group_t *g = &b->groups[b->group_of[index]];
    memset(C_out, 0, sizeof(*C_out));
    C_out->rows = b->A[index].rows;
    C_out->cols = b->B[index].cols;
    C_out->nnz = b->nnz[index];
    C_out->row_ptr = (int32_t *)b->crp_all.p + b->crp_off[index];
    C_out->col_idx = (int32_t *)g->c_ci.p + b->base[index];
    C_out->values = (float *)g->c_v.p + b->base[index];
    C_out->dtype = RVSP_DTYPE_FP32;
    C_out->format = RVSP_FORMAT_CSR;
    C_out->owns_data = 0;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_batch_copy_result(rvsp_spgemm_batch_t b, int32_t index,
                                            rvsp_csr_matrix_t *C)
{
    if (b == NULL || C == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (C->row_ptr == NULL || C->col_idx == NULL || C->values == NULL)
        return RVSP_ERROR_NULL_POINTER;
    rvsp_csr_matrix_t V;
    rvsp_status_t st = rvsp_spgemm_batch_get_result(b, index, &V);
    if (st != RVSP_SUCCESS)
        return st;
    if (C->rows != V.rows || C->cols != V.cols || C->nnz < V.nnz)
        return RVSP_ERROR_INVALID_ARGUMENT;
    cudaError_t e = cudaMemcpyAsync(C->row_ptr, V.row_ptr, ((size_t)V.rows + 1) * sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess && V.nnz > 0)
        e = cudaMemcpyAsync(C->col_idx, V.col_idx, (size_t)V.nnz * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess && V.nnz > 0)
        e = cudaMemcpyAsync(C->values, V.values, (size_t)V.nnz * sizeof(float),
                            cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
        return rvsp_map_cuda(e);
    return rvsp_spgemm_batch_synchronize(b);
}

rvsp_status_t rvsp_spgemm_batch_get_stats(rvsp_spgemm_batch_t b, int32_t *groups_out,
                                          int64_t *ops_out, int32_t *merge_policy_out,
                                          int32_t *graph_nodes_out)
{
    if (b == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (groups_out)
        *groups_out = b->ngroups;
    if (ops_out)
        *ops_out = b->total_ops;
    if (merge_policy_out)
        *merge_policy_out = b->merge_policy;
    if (graph_nodes_out) {
        size_t nodes = 0;
        if (b->graph && cudaGraphGetNodes(b->graph, NULL, &nodes) != cudaSuccess)
            nodes = 0;
        *graph_nodes_out = (int32_t)nodes;
    }
    return RVSP_SUCCESS;
}
