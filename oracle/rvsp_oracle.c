/*
 * CPU oracle for FP32 CSR SpGEMM.  TEST INFRASTRUCTURE ONLY: used by tests,
 * the smoke check and the benchmark's CPU-baseline leg as the checker, never
 * by the product library.
 *
 * Each function restates the behaviour of one reference function of
 * merledu/rv-sparse (paths relative to that project):
 *
 *   orc_csr_check       src/kernels/spgemm/rvsp_support.c:37-126
 *   orc_symbolic_count  src/kernels/spgemm/rvsp_symbolic.c:13-86
 *   orc_symbolic_fill   src/kernels/spgemm/rvsp_symbolic.c:91-137 and the
 *                       column sort of src/kernels/spgemm/rvsp_sort.h:106-122
 *                       (any correct ascending sort gives the same result,
 *                       the columns of a row being distinct)
 *   orc_numeric_f32     src/kernels/spgemm/gustavson_core_f32.inc:18-64 with
 *                       the scalar accumulate of accum_scalar_f32.c:20-71
 *
 * Arithmetic.  The reference is compiled with -std=c11, under which GCC does
 * not contract acc += a * b into a fused multiply-add, so each term is rounded
 * twice: p = fl(a * b), acc = fl(acc + p).  The accumulator of every output
 * entry starts at +0.0f (spgemm_descr.c:343, re-zeroed in
 * gustavson_core_f32.inc:61) and terms arrive in ascending A-nonzero order.
 * This file is built with -ffp-contract=off so the same two roundings happen
 * here.  orc_numeric_f64 is an independent FP64 accumulation used as the
 * high-precision reference for relative-error checks.
 */
#include "rvsp_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

int orc_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                  const int32_t *col_idx, int32_t *bad_row_out)
{
    if (bad_row_out)
        *bad_row_out = -1;
    if (rows < 0 || cols < 0 || row_ptr == NULL || row_ptr[0] != 0)
        return ORC_CSR_BAD_ROW_PTR;

    for (int32_t r = 0; r < rows; r++) {
        const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
        if (hi < lo) {
            if (bad_row_out)
                *bad_row_out = r;
            return ORC_CSR_BAD_ROW_PTR;
        }
        if (hi == lo)
            continue;
        if (col_idx == NULL)
            return ORC_CSR_BAD_ROW_PTR;
        int32_t last = -1;
        for (int32_t p = lo; p < hi; p++) {
            const int32_t c = col_idx[p];
            int code = ORC_CSR_OK;
            if (c < 0 || c >= cols)
                code = ORC_CSR_COL_OUT_OF_RANGE;
            else if (c == last)
                code = ORC_CSR_DUPLICATE;
            else if (c < last)
                code = ORC_CSR_UNSORTED;
            if (code != ORC_CSR_OK) {
                if (bad_row_out)
                    *bad_row_out = r;
                return code;
            }
            last = c;
        }
    }
    return ORC_CSR_OK;
}

int orc_symbolic_count(int32_t a_rows, int32_t b_cols,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx,
                       int32_t *c_row_ptr, int64_t *op_counts,
                       int64_t *total_nnz)
{
    /* stamp[c] == row + 1 marks column c as seen in the current row, which
     * needs no clearing between rows. */
    int32_t *stamp = (int32_t *)calloc((size_t)(b_cols > 0 ? b_cols : 1), sizeof(int32_t));
    if (!stamp)
        return -6;

    int64_t total = 0;
    for (int32_t r = 0; r < a_rows; r++) {
        int64_t ops = 0;
        int32_t distinct = 0;
        for (int32_t p = a_row_ptr[r]; p < a_row_ptr[r + 1]; p++) {
            const int32_t k = a_col_idx[p];
            ops += b_row_ptr[k + 1] - b_row_ptr[k];
            for (int32_t q = b_row_ptr[k]; q < b_row_ptr[k + 1]; q++) {
                const int32_t c = b_col_idx[q];
                if (stamp[c] != r + 1) {
                    stamp[c] = r + 1;
                    distinct++;
                }
            }
        }
        if (op_counts)
            op_counts[r] = ops;
        c_row_ptr[r] = distinct;
        total += distinct;
        if (total > INT32_MAX) {
            free(stamp);
            return -6;
        }
    }
    free(stamp);

    int32_t run = 0;
    for (int32_t r = 0; r < a_rows; r++) {
        const int32_t n = c_row_ptr[r];
        c_row_ptr[r] = run;
        run += n;
    }
    c_row_ptr[a_rows] = run;
    if (total_nnz)
        *total_nnz = total;
    return 0;
}

static int cmp_i32(const void *x, const void *y)
{
    const int32_t a = *(const int32_t *)x, b = *(const int32_t *)y;
    return (a > b) - (a < b);
}

void orc_symbolic_fill(int32_t a_rows, int32_t b_cols,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx,
                       const int32_t *c_row_ptr, int32_t *c_col_idx)
{
    int32_t *stamp = (int32_t *)calloc((size_t)(b_cols > 0 ? b_cols : 1), sizeof(int32_t));
    if (!stamp)
        return;
    for (int32_t r = 0; r < a_rows; r++) {
        int32_t *out = c_col_idx + c_row_ptr[r];
        int32_t n = 0;
        for (int32_t p = a_row_ptr[r]; p < a_row_ptr[r + 1]; p++) {
            const int32_t k = a_col_idx[p];
            for (int32_t q = b_row_ptr[k]; q < b_row_ptr[k + 1]; q++) {
                const int32_t c = b_col_idx[q];
                if (stamp[c] != r + 1) {
                    stamp[c] = r + 1;
                    out[n++] = c;
                }
            }
        }
        qsort(out, (size_t)n, sizeof(int32_t), cmp_i32);
    }
    free(stamp);
}

void orc_numeric_f32_rows(int32_t row_begin, int32_t row_end,
                          const int32_t *a_row_ptr, const int32_t *a_col_idx,
                          const float *a_values,
                          const int32_t *b_row_ptr, const int32_t *b_col_idx,
                          const float *b_values,
                          const int32_t *c_row_ptr, const int32_t *c_col_idx,
                          float *c_values, float *acc)
{
    for (int32_t r = row_begin; r < row_end; r++) {
        for (int32_t p = a_row_ptr[r]; p < a_row_ptr[r + 1]; p++) {
            const int32_t k = a_col_idx[p];
            const float a = a_values[p];
            for (int32_t q = b_row_ptr[k]; q < b_row_ptr[k + 1]; q++) {
                const float term = a * b_values[q];      /* rounded once   */
                acc[b_col_idx[q]] = acc[b_col_idx[q]] + term; /* and again */
            }
        }
        for (int32_t e = c_row_ptr[r]; e < c_row_ptr[r + 1]; e++) {
            c_values[e] = acc[c_col_idx[e]];
            acc[c_col_idx[e]] = 0.0f;
        }
    }
}

void orc_numeric_f32(int32_t a_rows, int32_t b_cols,
                     const int32_t *a_row_ptr, const int32_t *a_col_idx,
                     const float *a_values,
                     const int32_t *b_row_ptr, const int32_t *b_col_idx,
                     const float *b_values,
                     const int32_t *c_row_ptr, const int32_t *c_col_idx,
                     float *c_values)
{
    float *acc = (float *)calloc((size_t)(b_cols > 0 ? b_cols : 1), sizeof(float));
    if (!acc)
        return;
    orc_numeric_f32_rows(0, a_rows, a_row_ptr, a_col_idx, a_values, b_row_ptr,
                         b_col_idx, b_values, c_row_ptr, c_col_idx, c_values, acc);
    free(acc);
}

void orc_numeric_f64(int32_t a_rows, int32_t b_cols,
                     const int32_t *a_row_ptr, const int32_t *a_col_idx,
                     const float *a_values,
                     const int32_t *b_row_ptr, const int32_t *b_col_idx,
                     const float *b_values,
                     const int32_t *c_row_ptr, const int32_t *c_col_idx,
                     double *c_values, double *c_abs_sum)
{
    const size_t n = (size_t)(b_cols > 0 ? b_cols : 1);
    double *acc = (double *)calloc(n, sizeof(double));
    double *mag = (double *)calloc(n, sizeof(double));
    if (!acc || !mag) {
        free(acc);
        free(mag);
        return;
    }
    for (int32_t r = 0; r < a_rows; r++) {
        for (int32_t p = a_row_ptr[r]; p < a_row_ptr[r + 1]; p++) {
            const int32_t k = a_col_idx[p];
            const double a = (double)a_values[p];
            for (int32_t q = b_row_ptr[k]; q < b_row_ptr[k + 1]; q++) {
                /* a float times a float is exact in double */
                const double t = a * (double)b_values[q];
                acc[b_col_idx[q]] += t;
                mag[b_col_idx[q]] += t < 0 ? -t : t;
            }
        }
        for (int32_t e = c_row_ptr[r]; e < c_row_ptr[r + 1]; e++) {
            c_values[e] = acc[c_col_idx[e]];
            if (c_abs_sum)
                c_abs_sum[e] = mag[c_col_idx[e]];
            acc[c_col_idx[e]] = 0.0;
            mag[c_col_idx[e]] = 0.0;
        }
    }
    free(acc);
    free(mag);
}
