/*
 * CPU oracle for the FP64 and INT8 -> INT32 products.  TEST INFRASTRUCTURE
 * ONLY: used by tests as the checker, never by the product library.
 *
 * orc_spgemm_f64 / orc_spgemm_i8 restate the numeric passes of the legacy
 * scalar kernels of merledu/rv-sparse (paths relative to that project):
 *   src/kernels/spgemm/legacy/csr_scalar_f64.c:196-262
 *   src/kernels/spgemm/legacy/csr_scalar_i8.c:137-185
 * per row: a dense accumulator over B's columns, entries touched in product
 * order set to zero on first touch, then acc += a * b (FP64: two roundings,
 * this file is built with -ffp-contract=off as the reference's -std=c11
 * build contracts nothing; INT8: int32 products summed in int32, wrapping);
 * the touched columns sorted ascending; an entry is stored only when its sum
 * is not zero.  Inputs must be canonical CSR (the GPU path requires it).
 * Outputs are malloc'd (release with orc_free); returns 0, or -3 when out of
 * memory.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rvsp_oracle.h"

static int cmp_i32(const void *a, const void *b)
{
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* elem: 8 (double in, double out) or 1 (int8 in, int32 out) */
static int typed(int elem, int32_t a_rows, int32_t b_cols, const int32_t *a_rp,
                 const int32_t *a_ci, const void *a_v, const int32_t *b_rp,
                 const int32_t *b_ci, const void *b_v, int32_t **rp_out, int32_t **ci_out,
                 void **v_out, int64_t *nnz_out)
{
    const size_t bc = (size_t)(b_cols > 0 ? b_cols : 1);
    double *accd = elem == 8 ? (double *)malloc(bc * sizeof(double)) : NULL;
    int32_t *acci = elem == 1 ? (int32_t *)malloc(bc * sizeof(int32_t)) : NULL;
    uint8_t *mark = (uint8_t *)calloc(bc, 1);
    int32_t *touched = (int32_t *)malloc(bc * sizeof(int32_t));
    int32_t *rp = (int32_t *)calloc((size_t)a_rows + 1, sizeof(int32_t));
    size_t cap = 1024, n = 0;
    int32_t *ci = (int32_t *)malloc(cap * sizeof(int32_t));
    void *v = malloc(cap * (elem == 8 ? sizeof(double) : sizeof(int32_t)));
    if ((!accd && !acci) || !mark || !touched || !rp || !ci || !v)
        goto oom;
    for (int32_t row = 0; row < a_rows; row++) {
        int32_t nt = 0;
        for (int32_t p = a_rp[row]; p < a_rp[row + 1]; p++) {
            const int32_t k = a_ci[p];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++) {
                const int32_t col = b_ci[q];
                if (!mark[col]) {
                    mark[col] = 1;
                    if (elem == 8)
                        accd[col] = 0.0;
                    else
                        acci[col] = 0;
                    touched[nt++] = col;
                }
                if (elem == 8) {
                    accd[col] += ((const double *)a_v)[p] * ((const double *)b_v)[q];
                } else {
                    const int32_t prod = (int32_t)((const int8_t *)a_v)[p] *
                                         (int32_t)((const int8_t *)b_v)[q];
                    acci[col] = (int32_t)((uint32_t)acci[col] + (uint32_t)prod);
                }
            }
        }
        qsort(touched, (size_t)nt, sizeof(int32_t), cmp_i32);
        for (int32_t i = 0; i < nt; i++) {
            const int32_t col = touched[i];
            mark[col] = 0;
            const int keep = elem == 8 ? accd[col] != 0.0 : acci[col] != 0;
            if (!keep)
                continue;
            if (n == cap) {
                cap *= 2;
                int32_t *ci2 = (int32_t *)realloc(ci, cap * sizeof(int32_t));
                void *v2 = realloc(v, cap * (elem == 8 ? sizeof(double) : sizeof(int32_t)));
                if (ci2)
                    ci = ci2;
                if (v2)
                    v = v2;
                if (!ci2 || !v2)
                    goto oom;
            }
            ci[n] = col;
            if (elem == 8)
                ((double *)v)[n] = accd[col];
            else
                ((int32_t *)v)[n] = acci[col];
            n++;
        }
        rp[row + 1] = (int32_t)n;
    }
    free(accd);
    free(acci);
    free(mark);
    free(touched);
    *rp_out = rp;
    *ci_out = ci;
    *v_out = v;
    *nnz_out = (int64_t)n;
    return 0;
oom:
    free(accd);
    free(acci);
    free(mark);
    free(touched);
    free(rp);
    free(ci);
    free(v);
    return -3;
}

int orc_spgemm_f64(int32_t a_rows, int32_t b_cols, const int32_t *a_rp, const int32_t *a_ci,
                   const double *a_v, const int32_t *b_rp, const int32_t *b_ci,
                   const double *b_v, int32_t **rp_out, int32_t **ci_out, double **v_out,
                   int64_t *nnz_out)
{
    return typed(8, a_rows, b_cols, a_rp, a_ci, a_v, b_rp, b_ci, b_v, rp_out, ci_out,
                 (void **)v_out, nnz_out);
}

int orc_spgemm_i8(int32_t a_rows, int32_t b_cols, const int32_t *a_rp, const int32_t *a_ci,
                  const int8_t *a_v, const int32_t *b_rp, const int32_t *b_ci,
                  const int8_t *b_v, int32_t **rp_out, int32_t **ci_out, int32_t **v_out,
                  int64_t *nnz_out)
{
    return typed(1, a_rows, b_cols, a_rp, a_ci, a_v, b_rp, b_ci, b_v, rp_out, ci_out,
                 (void **)v_out, nnz_out);
}
