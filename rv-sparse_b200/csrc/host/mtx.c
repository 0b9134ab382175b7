/*
 * Matrix Market reader: a coordinate file to canonical CSR.
 *
 * Follows the reference's assemble_csr_matrix
 * (tools/src/mtx_to_csr_formatter.c:148-325) token for token:
 *   - the first line (read as fgets does into a 2048-byte buffer) is the
 *     banner; "pattern" gives every entry the value 1.0f and "symmetric"
 *     mirrors every off-diagonal entry (:37-58, :248-273);
 *   - further lines starting with '%' are skipped; the first other line holds
 *     "M N L" (:26-35, :171-180);
 *   - then up to L entries "%d %d %f" (or "%d %d"), 1-based, read as fscanf
 *     reads them, stopping at the first entry that does not convert (:196-219).
 * The entries are then made canonical on the GPU (rvsp_cuda_coo_to_csr:
 * rows sorted by column, repeated entries summed in file order, mirrors
 * after all stored entries), which reproduces the reference's values bit for
 * bit.  Differences: an index outside 1..M / 1..N is rejected with
 * RVSP_ERROR_INVALID_CSR (the reference writes out of bounds), and the
 * result carries N as its column count (the reference's CSR struct has none).
 *
 * The entries are parsed on all host cores: the text after the size line is
 * cut at whitespace into one piece per thread, each thread counts its tokens,
 * and then converts them knowing each token's global index (entry = index /
 * fields, field = index % fields).  That equals fscanf's reading whenever each
 * conversion consumes its whole token; if any does not (say "1.5" read as an
 * integer), the file is read again by a sequential scanner that advances
 * exactly as fscanf does.
 */
#include <ctype.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "rvsp_internal.h"

#define MTX_LINE 2048 /* the reference's fgets buffer */
#define MTX_PARALLEL_MIN ((size_t)4 << 20)
#define MTX_MAX_THREADS 64

/* fgets(buf, MTX_LINE, f) on an in-memory text. */
static int next_line(const char *t, size_t len, size_t *pos, char *buf)
{
    size_t n = 0;
    if (*pos >= len)
        return 0;
    while (*pos < len && n < MTX_LINE - 1) {
        const char ch = t[(*pos)++];
        buf[n++] = ch;
        if (ch == '\n')
            break;
    }
    buf[n] = '\0';
    return 1;
}

/* parse_banner (mtx_to_csr_formatter.c:37-58). */
static void parse_banner(const char *buf, int *is_pattern, int *is_symmetric)
{
    char object[64], format[64], field[64], symmetry[64];
    *is_pattern = 0;
    *is_symmetric = 0;
    if (strncmp(buf, "%%MatrixMarket", 14) != 0)
        return;
    if (sscanf(buf, "%%%%MatrixMarket %63s %63s %63s %63s", object, format, field,
               symmetry) < 4)
        return;
    if (strcmp(field, "pattern") == 0)
        *is_pattern = 1;
    if (strcmp(symmetry, "symmetric") == 0)
        *is_symmetric = 1;
}

/* One conversion as fscanf's %d / %f: skip white space, convert, advance by
 * what the conversion consumed.  0 when nothing converts. */
static int scan_int(const char *t, size_t len, size_t *pos, int *out)
{
    char *end;
    while (*pos < len && isspace((unsigned char)t[*pos]))
        (*pos)++;
    if (*pos >= len)
        return 0;
    const long v = strtol(t + *pos, &end, 10);
    if (end == t + *pos)
        return 0;
    *pos = (size_t)(end - t);
    *out = (int)v;
    return 1;
}

static int scan_float(const char *t, size_t len, size_t *pos, float *out)
{
    char *end;
    while (*pos < len && isspace((unsigned char)t[*pos]))
        (*pos)++;
    if (*pos >= len)
        return 0;
    const float v = strtof(t + *pos, &end);
    if (end == t + *pos)
        return 0;
    *pos = (size_t)(end - t);
    *out = v;
    return 1;
}

typedef struct {
    const char *t;
    size_t beg, end;       /* this thread's piece */
    int fields;            /* 2 (pattern) or 3 */
    int64_t first;         /* global index of the piece's first token */
    int64_t tokens;        /* tokens in the piece (phase 1) */
    int64_t limit;         /* entries wanted (L, capped) */
    int64_t fail;          /* first entry that did not convert, or limit */
    int irregular;         /* a conversion stopped inside its token */
    int32_t *row, *col;
    float *val;
} piece_t;

static void *count_tokens(void *arg)
{
    piece_t *p = (piece_t *)arg;
    int64_t n = 0;
    size_t i = p->beg;
    while (i < p->end) {
        while (i < p->end && isspace((unsigned char)p->t[i]))
            i++;
        if (i >= p->end)
            break;
        n++;
        while (i < p->end && !isspace((unsigned char)p->t[i]))
            i++;
    }
    p->tokens = n;
    return NULL;
}

static void *convert_tokens(void *arg)
{
    piece_t *p = (piece_t *)arg;
    int64_t g = p->first;
    size_t i = p->beg;
    p->fail = p->limit;
    p->irregular = 0;
    while (i < p->end) {
        while (i < p->end && isspace((unsigned char)p->t[i]))
            i++;
        if (i >= p->end)
            break;
        size_t j = i;
        while (j < p->end && !isspace((unsigned char)p->t[j]))
            j++;
        const int64_t e = g / p->fields;
        const int f = (int)(g % p->fields);
        if (e >= p->limit || e >= p->fail)
            break;
        char *stop;
        if (f < 2) {
            const long v = strtol(p->t + i, &stop, 10);
            if (stop == p->t + i) {
                p->fail = e;
                break;
            }
            if (stop != p->t + j)
                p->irregular = 1;
            if (f == 0)
                p->row[e] = (int32_t)v - 1;
            else
                p->col[e] = (int32_t)v - 1;
        } else {
            const float v = strtof(p->t + i, &stop);
            if (stop == p->t + i) {
                p->fail = e;
                break;
            }
            if (stop != p->t + j)
                p->irregular = 1;
            p->val[e] = v;
        }
        g++;
        i = j;
    }
    return NULL;
}

/* Sequential reading of the entries, fscanf's way.  Returns entries read. */
static int64_t read_entries_seq(const char *t, size_t len, size_t pos, int pattern,
                                int64_t limit, int32_t *row, int32_t *col, float *val)
{
    int64_t n = 0;
    for (; n < limit; n++) {
        int r, c;
        float v = 1.0f;
        if (!scan_int(t, len, &pos, &r) || !scan_int(t, len, &pos, &c))
            break;
        if (!pattern && !scan_float(t, len, &pos, &v))
            break;
        row[n] = r - 1;
        col[n] = c - 1;
        val[n] = v;
    }
    return n;
}

static int64_t read_entries(const char *t, size_t len, size_t pos, int pattern,
                            int64_t limit, int32_t *row, int32_t *col, float *val)
{
    const int fields = pattern ? 2 : 3;
    long nproc = sysconf(_SC_NPROCESSORS_ONLN);
    int nt = nproc > 0 ? (int)nproc : 1;
    if (nt > MTX_MAX_THREADS)
        nt = MTX_MAX_THREADS;
    if (len - pos < MTX_PARALLEL_MIN || nt < 2)
        return read_entries_seq(t, len, pos, pattern, limit, row, col, val);
    piece_t pc[MTX_MAX_THREADS];
    pthread_t th[MTX_MAX_THREADS];
    size_t b = pos;
    for (int i = 0; i < nt; i++) {
        size_t e = i == nt - 1 ? len : pos + (len - pos) / (size_t)nt * (size_t)(i + 1);
        while (e < len && !isspace((unsigned char)t[e]))
            e++;
        if (e < b)
            e = b;
        pc[i] = (piece_t){t, b, e, fields, 0, 0, limit, limit, 0, row, col, val};
        b = e;
    }
    int started = 0;
    for (; started < nt; started++)
        if (pthread_create(&th[started], NULL, count_tokens, &pc[started]) != 0)
            break;
    for (int i = 0; i < started; i++)
        pthread_join(th[i], NULL);
    if (started < nt)
        return read_entries_seq(t, len, pos, pattern, limit, row, col, val);
    int64_t g = 0;
    for (int i = 0; i < nt; i++) {
        pc[i].first = g;
        g += pc[i].tokens;
    }
    const int64_t total_tokens = g;
    for (started = 0; started < nt; started++)
        if (pthread_create(&th[started], NULL, convert_tokens, &pc[started]) != 0)
            break;
    for (int i = 0; i < started; i++)
        pthread_join(th[i], NULL);
    if (started < nt)
        return read_entries_seq(t, len, pos, pattern, limit, row, col, val);
    int64_t n = total_tokens / fields;
    if (n > limit)
        n = limit;
    for (int i = 0; i < nt; i++) {
        if (pc[i].irregular)
            return read_entries_seq(t, len, pos, pattern, limit, row, col, val);
        if (pc[i].fail < n)
            n = pc[i].fail;
    }
    if (pattern)
        for (int64_t k = 0; k < n; k++)
            val[k] = 1.0f;
    return n;
}

/* COO (device) to CSR in the requested memory space. */
static rvsp_status_t finish(int32_t M, int32_t N, int64_t n, int symmetric, const int32_t *row,
                            const int32_t *col, const float *val, rvsp_memory_space_t space,
                            rvsp_csr_matrix_t *out)
{
    int32_t *d_row = NULL, *d_col = NULL, *d_rp = NULL, *c_col = NULL;
    float *d_val = NULL, *c_val = NULL;
    int32_t nnz = 0;
    const size_t nb = (size_t)(n > 0 ? n : 1);
    rvsp_status_t st = RVSP_SUCCESS;
    cudaError_t e = cudaMalloc((void **)&d_row, nb * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_col, nb * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_val, nb * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_rp, ((size_t)M + 1) * sizeof(int32_t));
    if (e == cudaSuccess && n > 0) {
        e = cudaMemcpy(d_row, row, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_col, col, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(d_val, val, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        st = rvsp_map_cuda(e);
        goto done;
    }
    st = rvsp_cuda_coo_to_csr(NULL, M, N, n, symmetric, d_row, d_col, d_val, d_rp, &c_col,
                              &c_val, &nnz);
    if (st != RVSP_SUCCESS)
        goto done;
    memset(out, 0, sizeof(*out));
    out->rows = M;
    out->cols = N;
    out->nnz = nnz;
    out->dtype = RVSP_DTYPE_FP32;
    out->format = RVSP_FORMAT_CSR;
    if (space == RVSP_MEM_DEVICE) {
        out->row_ptr = d_rp;
        out->col_idx = c_col;
        out->values = c_val;
        out->owns_data = 2;
        d_rp = NULL;
        c_col = NULL;
        c_val = NULL;
    } else {
        const size_t cn = (size_t)(nnz > 0 ? nnz : 1);
        int32_t *h_rp = (int32_t *)rvsp_malloc(((size_t)M + 1) * sizeof(int32_t));
        int32_t *h_col = (int32_t *)rvsp_malloc(cn * sizeof(int32_t));
        float *h_val = (float *)rvsp_malloc(cn * sizeof(float));
        if (!h_rp || !h_col || !h_val) {
            free(h_rp);
            free(h_col);
            free(h_val);
            memset(out, 0, sizeof(*out));
            st = RVSP_ERROR_ALLOCATION_FAILED;
            goto done;
        }
        e = cudaMemcpy(h_rp, d_rp, ((size_t)M + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && nnz > 0)
            e = cudaMemcpy(h_col, c_col, (size_t)nnz * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && nnz > 0)
            e = cudaMemcpy(h_val, c_val, (size_t)nnz * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            free(h_rp);
            free(h_col);
            free(h_val);
            memset(out, 0, sizeof(*out));
            st = rvsp_map_cuda(e);
            goto done;
        }
        out->row_ptr = h_rp;
        out->col_idx = h_col;
        out->values = h_val;
        out->owns_data = 1;
    }
done:
    cudaFree(d_row);
    cudaFree(d_col);
    cudaFree(d_val);
    cudaFree(d_rp);
    cudaFree(c_col);
    cudaFree(c_val);
    return st;
}

rvsp_status_t rvsp_csr_parse_mtx(const char *text, size_t len, rvsp_memory_space_t space,
                                 rvsp_csr_matrix_t *out)
{
    if (!text || !out)
        return RVSP_ERROR_NULL_POINTER;
    memset(out, 0, sizeof(*out)); /* every failure leaves out empty */
    if (space != RVSP_MEM_HOST && space != RVSP_MEM_DEVICE)
        return RVSP_ERROR_INVALID_ARGUMENT;
    /* a NUL-terminated copy: strtol / strtof must not run past the text */
    char *t = (char *)rvsp_malloc(len + 1);
    if (!t)
        return RVSP_ERROR_ALLOCATION_FAILED;
    memcpy(t, text, len);
    t[len] = '\0';
    char buf[MTX_LINE];
    size_t pos = 0;
    int pattern = 0, symmetric = 0;
    rvsp_status_t st = RVSP_SUCCESS;
    buf[0] = '\0';
    if (next_line(t, len, &pos, buf))
        parse_banner(buf, &pattern, &symmetric);
    while (next_line(t, len, &pos, buf))
        if (buf[0] != '%')
            break;
    int M, N, L;
    if (sscanf(buf, "%d %d %d", &M, &N, &L) != 3 || M < 0 || N < 0 || L < 0) {
        free(t);
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    /* an entry takes at least fields tokens and separators */
    const int fields = pattern ? 2 : 3;
    int64_t limit = L;
    const int64_t fit = (int64_t)((len - pos) / (size_t)(2 * fields)) + 1;
    if (limit > fit)
        limit = fit;
    const size_t nb = (size_t)(limit > 0 ? limit : 1);
    int32_t *row = (int32_t *)rvsp_malloc(nb * sizeof(int32_t));
    int32_t *col = (int32_t *)rvsp_malloc(nb * sizeof(int32_t));
    float *val = (float *)rvsp_malloc(nb * sizeof(float));
    if (!row || !col || !val) {
        st = RVSP_ERROR_ALLOCATION_FAILED;
    } else {
        const int64_t n = read_entries(t, len, pos, pattern, limit, row, col, val);
        st = finish(M, N, n, symmetric, row, col, val, space, out);
    }
    free(row);
    free(col);
    free(val);
    free(t);
    return st;
}

rvsp_status_t rvsp_csr_read_mtx(const char *path, rvsp_memory_space_t space,
                                rvsp_csr_matrix_t *out)
{
    if (!path || !out)
        return RVSP_ERROR_NULL_POINTER;
    memset(out, 0, sizeof(*out)); /* every failure leaves out empty */
    FILE *f = fopen(path, "rb");
    if (!f)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (fseek(f, 0, SEEK_END) != 0) {
        fclose(f);
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    const long size = ftell(f);
    if (size < 0 || fseek(f, 0, SEEK_SET) != 0) {
        fclose(f);
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    char *t = (char *)rvsp_malloc((size_t)size + 1);
    if (!t) {
        fclose(f);
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    const size_t got = fread(t, 1, (size_t)size, f);
    fclose(f);
    const rvsp_status_t st = rvsp_csr_parse_mtx(t, got, space, out);
    free(t);
    return st;
}
