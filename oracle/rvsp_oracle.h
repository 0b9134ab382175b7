/*
 * CPU oracle for FP32 CSR SpGEMM, C = A * B.  TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference scalar backend of
 * merledu/rv-sparse: symbolic count, sorted symbolic fill, and the Gustavson
 * numeric pass with a dense accumulator.  It exists to check the CUDA path and
 * is never linked into, loaded by, or called from the product library.  Only
 * tests, the smoke check and the CPU-baseline leg of the benchmark use it.
 *
 * Parity is pinned two ways: against the hand-computed fixtures of the
 * reference test suite (tests/csr_fixtures.h:42-153) and bit-for-bit against
 * the reference library itself, compiled from its sources into
 * oracle/_ref/librvsp_ref.so.
 */
#ifndef RVSP_ORACLE_H
#define RVSP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same codes and order as rvsp_csr_status_t (src/kernels/spgemm/rvsp_spgemm.h:38-45). */
enum {
    ORC_CSR_OK = 0,
    ORC_CSR_BAD_ROW_PTR = 1,
    ORC_CSR_COL_OUT_OF_RANGE = 2,
    ORC_CSR_UNSORTED = 3,
    ORC_CSR_DUPLICATE = 4
};

int orc_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                  const int32_t *col_idx, int32_t *bad_row_out);

/* Returns 0, or -6 (allocation failed) when nnz(C) exceeds INT32_MAX. */
int orc_symbolic_count(int32_t a_rows, int32_t b_cols,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx,
                       int32_t *c_row_ptr, int64_t *op_counts,
                       int64_t *total_nnz);

void orc_symbolic_fill(int32_t a_rows, int32_t b_cols,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx,
                       const int32_t *c_row_ptr, int32_t *c_col_idx);

void orc_numeric_f32(int32_t a_rows, int32_t b_cols,
                     const int32_t *a_row_ptr, const int32_t *a_col_idx,
                     const float *a_values,
                     const int32_t *b_row_ptr, const int32_t *b_col_idx,
                     const float *b_values,
                     const int32_t *c_row_ptr, const int32_t *c_col_idx,
                     float *c_values);

void orc_numeric_f64(int32_t a_rows, int32_t b_cols,
                     const int32_t *a_row_ptr, const int32_t *a_col_idx,
                     const float *a_values,
                     const int32_t *b_row_ptr, const int32_t *b_col_idx,
                     const float *b_values,
                     const int32_t *c_row_ptr, const int32_t *c_col_idx,
                     double *c_values, double *c_abs_sum);

/* Numeric pass over a row range [row_begin, row_end); used to split work
 * across host threads.  acc must hold b_cols zeroed floats and is left zeroed. */
void orc_numeric_f32_rows(int32_t row_begin, int32_t row_end,
                          const int32_t *a_row_ptr, const int32_t *a_col_idx,
                          const float *a_values,
                          const int32_t *b_row_ptr, const int32_t *b_col_idx,
                          const float *b_values,
                          const int32_t *c_row_ptr, const int32_t *c_col_idx,
                          float *c_values, float *acc);

/* Matrix Market coordinate text to canonical CSR (mtx_oracle.c).  Returns 0,
 * -1 for a malformed size line, -2 for an index out of range, -3 when out of
 * memory.  The three arrays are malloc'd: release them with orc_free. */
int orc_mtx_to_csr(const char *text, size_t len, int32_t *rows_out, int32_t *cols_out,
                   int64_t *nnz_out, int32_t **row_ptr_out, int32_t **col_idx_out,
                   float **values_out);
void orc_free(void *p);

/* FP64 and INT8 -> INT32 products of the legacy scalar kernels
 * (typed_oracle.c).  0, or -3 when out of memory; outputs for orc_free. */
int orc_spgemm_f64(int32_t a_rows, int32_t b_cols, const int32_t *a_rp, const int32_t *a_ci,
                   const double *a_v, const int32_t *b_rp, const int32_t *b_ci,
                   const double *b_v, int32_t **rp_out, int32_t **ci_out, double **v_out,
                   int64_t *nnz_out);
int orc_spgemm_i8(int32_t a_rows, int32_t b_cols, const int32_t *a_rp, const int32_t *a_ci,
                  const int8_t *a_v, const int32_t *b_rp, const int32_t *b_ci,
                  const int8_t *b_v, int32_t **rp_out, int32_t **ci_out, int32_t **v_out,
                  int64_t *nnz_out);

#ifdef __cplusplus
}
#endif

#endif
