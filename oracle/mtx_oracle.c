/*
 * CPU oracle for the Matrix Market reader.  TEST INFRASTRUCTURE ONLY: used by
 * tests and the benchmark's CPU-baseline leg as the checker, never by the
 * product library.
 *
 * orc_mtx_to_csr restates assemble_csr_matrix of merledu/rv-sparse
 * (tools/src/mtx_to_csr_formatter.c, paths relative to that project) step by
 * step, reading the text through a memory stream with the same stdio calls:
 *   banner       first line by fgets into 2048 bytes; "pattern" / "symmetric"
 *                (:37-58, :160-164)
 *   comments     further lines while they start with '%' (:26-35)
 *   size         sscanf "%d %d %d" of the first other line (:171-177)
 *   entries      up to L entries by fscanf "%d %d" or "%d %d %f", stopping at
 *                the first that does not convert; 1-based (:196-219)
 *   symmetric    the mirror of every off-diagonal entry appended after all
 *                stored entries, in stored order (:248-273)
 *   scatter      entries to their rows in that order (:275-311)
 *   canonicalise each row sorted by column, equal columns kept in order
 *                (glibc 2.39's qsort is a merge sort for these sizes; here
 *                the order is made explicit), runs summed from their first
 *                value: acc = v0, acc += v ... (:67-146)
 * It checks what the reference leaves undefined: an index outside 1..M x
 * 1..N (or a mirror outside it) returns -2.
 */
#define _POSIX_C_SOURCE 200809L

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rvsp_oracle.h"

typedef struct {
    int32_t col;
    int64_t order; /* position in the COO list: stable sort key */
    float val;
} orc_cv_t;

static int cmp_cv(const void *a, const void *b)
{
    const orc_cv_t *x = (const orc_cv_t *)a, *y = (const orc_cv_t *)b;
    if (x->col != y->col)
        return (x->col > y->col) - (x->col < y->col);
    return (x->order > y->order) - (x->order < y->order);
}

void orc_free(void *p) { free(p); }

int orc_mtx_to_csr(const char *text, size_t len, int32_t *rows_out, int32_t *cols_out,
                   int64_t *nnz_out, int32_t **row_ptr_out, int32_t **col_idx_out,
                   float **values_out)
{
    *row_ptr_out = NULL;
    *col_idx_out = NULL;
    *values_out = NULL;
    FILE *f = fmemopen((void *)text, len, "r");
    if (!f)
        return -3;
    char buf[2048];
    int is_pattern = 0, is_symmetric = 0;
    buf[0] = '\0';
    if (fgets(buf, sizeof(buf), f) != NULL) {
        char object[64], format[64], field[64], symmetry[64];
        if (strncmp(buf, "%%MatrixMarket", 14) == 0 &&
            sscanf(buf, "%%%%MatrixMarket %63s %63s %63s %63s", object, format, field,
                   symmetry) >= 4) {
            is_pattern = strcmp(field, "pattern") == 0;
            is_symmetric = strcmp(symmetry, "symmetric") == 0;
        }
    }
    while (fgets(buf, sizeof(buf), f) != NULL)
        if (buf[0] != '%')
            break;
    int M, N, L;
    if (sscanf(buf, "%d %d %d", &M, &N, &L) != 3 || M < 0 || N < 0 || L < 0) {
        fclose(f);
        return -1;
    }
    const size_t cap = (size_t)L * (is_symmetric ? 2 : 1) + 1;
    int32_t *r = (int32_t *)malloc(cap * sizeof(int32_t));
    int32_t *c = (int32_t *)malloc(cap * sizeof(int32_t));
    float *v = (float *)malloc(cap * sizeof(float));
    if (!r || !c || !v) {
        free(r);
        free(c);
        free(v);
        fclose(f);
        return -3;
    }
    int64_t n = 0;
    for (int l = 0; l < L; l++) {
        int row, col;
        float val = 1.0f;
        if (is_pattern) {
            if (fscanf(f, "%d %d", &row, &col) != 2)
                break;
        } else {
            if (fscanf(f, "%d %d %f", &row, &col, &val) != 3)
                break;
        }
        r[n] = row - 1;
        c[n] = col - 1;
        v[n] = val;
        n++;
    }
    fclose(f);
    int bad = 0;
    for (int64_t k = 0; k < n; k++)
        if (r[k] < 0 || r[k] >= M || c[k] < 0 || c[k] >= N)
            bad = 1;
    if (!bad && is_symmetric) {
        const int64_t stored = n;
        for (int64_t k = 0; k < stored; k++) {
            if (r[k] != c[k]) {
                if (c[k] >= M || r[k] >= N)
                    bad = 1;
                r[n] = c[k];
                c[n] = r[k];
                v[n] = v[k];
                n++;
            }
        }
    }
    if (bad) {
        free(r);
        free(c);
        free(v);
        return -2;
    }
    int32_t *rp = (int32_t *)calloc((size_t)M + 1, sizeof(int32_t));
    orc_cv_t *e = (orc_cv_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(orc_cv_t));
    int32_t *ci = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    float *cv = (float *)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
    int64_t *cursor = (int64_t *)malloc(((size_t)M + 1) * sizeof(int64_t));
    if (!rp || !e || !ci || !cv || !cursor) {
        free(r);
        free(c);
        free(v);
        free(rp);
        free(e);
        free(ci);
        free(cv);
        free(cursor);
        return -3;
    }
    /* scatter in COO order */
    int64_t *start = cursor;
    for (int64_t k = 0; k < n; k++)
        rp[r[k] + 1]++;
    for (int32_t i = 0; i < M; i++)
        rp[i + 1] += rp[i];
    for (int32_t i = 0; i <= M; i++)
        start[i] = rp[i];
    for (int64_t k = 0; k < n; k++) {
        const int64_t d = start[r[k]]++;
        e[d].col = c[k];
        e[d].order = k;
        e[d].val = v[k];
    }
    /* canonicalise: sort each row by column, sum runs from their first value */
    int64_t w = 0;
    int32_t prev = 0;
    for (int32_t i = 0; i < M; i++) {
        const int32_t s0 = prev, s1 = rp[i + 1];
        prev = s1;
        qsort(e + s0, (size_t)(s1 - s0), sizeof(orc_cv_t), cmp_cv);
        int32_t t = s0;
        while (t < s1) {
            const int32_t col = e[t].col;
            float acc = e[t].val;
            t++;
            while (t < s1 && e[t].col == col) {
                acc += e[t].val;
                t++;
            }
            ci[w] = col;
            cv[w] = acc;
            w++;
        }
        rp[i + 1] = (int32_t)w;
    }
    free(r);
    free(c);
    free(v);
    free(e);
    free(cursor);
    *rows_out = M;
    *cols_out = N;
    *nnz_out = w;
    *row_ptr_out = rp;
    *col_idx_out = ci;
    *values_out = cv;
    return 0;
}
