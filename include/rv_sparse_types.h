/*
 * rv-sparse-b200: public types.
 *
 * Drop-in replacement for the types of merledu/rv-sparse
 * (include/rv_sparse_types.h:21-96 in that project).  Every enumerator keeps
 * its name and numeric value there, so code compiled against the reference
 * headers binds to this library unchanged; additions are appended after the
 * reference's last value and never renumber an existing one.
 */
#ifndef RV_SPARSE_TYPES_H
#define RV_SPARSE_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  -1..-6 are the reference codes (rv_sparse_types.h:21-30);
 * RVSP_ERROR_DEVICE is new: a CUDA call failed or a kernel reported an
 * internal error through its status word (never a fault). */
typedef enum {
    RVSP_SUCCESS = 0,
    RVSP_ERROR_NULL_POINTER = -1,
    RVSP_ERROR_INVALID_ARGUMENT = -2,
    RVSP_ERROR_INVALID_CSR = -3,
    RVSP_ERROR_UNSUPPORTED_DTYPE = -4,
    RVSP_ERROR_UNSUPPORTED_BACKEND = -5,
    RVSP_ERROR_ALLOCATION_FAILED = -6,
    RVSP_ERROR_DEVICE = -7
} rvsp_status_t;

/* Element types (rv_sparse_types.h:32-39). */
typedef enum {
    RVSP_DTYPE_INT8,
    RVSP_DTYPE_INT32,
    RVSP_DTYPE_BF16,
    RVSP_DTYPE_FP32,
    RVSP_DTYPE_FP64
} rvsp_dtype_t;

typedef enum {
    RVSP_FORMAT_CSR
} rvsp_format_t;

/* Backends (rv_sparse_types.h:46-51).  This library implements only
 * RVSP_BACKEND_CUDA; the three CPU backends report
 * RVSP_ERROR_UNSUPPORTED_BACKEND, as the reference does for a backend its
 * build lacks. */
typedef enum {
    RVSP_BACKEND_SCALAR,
    RVSP_BACKEND_SCALAR_UNROLL4,
    RVSP_BACKEND_RVV_INTRINSICS,
    RVSP_BACKEND_CUDA
} rvsp_backend_t;

/* CSR matrix (rv_sparse_types.h:53-67), same field order and types.
 * owns_data: 0 caller-owned, 1 library-owned host arrays (free),
 * 2 library-owned device arrays (cudaFree). */
typedef struct {
    int32_t rows;
    int32_t cols;
    int32_t nnz;

    int32_t *row_ptr;
    int32_t *col_idx;
    void *values;

    rvsp_dtype_t dtype;
    rvsp_format_t format;

    int owns_data;
} rvsp_csr_matrix_t;

typedef struct {
    rvsp_backend_t backend;
    rvsp_dtype_t input_dtype;
    rvsp_dtype_t output_dtype;
} rvsp_spgemm_options_t;

/* Opaque descriptor holding the analysed structure between the structure
 * and numeric phases (rv_sparse_types.h:82). */
typedef struct rvsp_spgemm_descr *rvsp_spgemm_descr_t;

/* Strategies (rv_sparse_types.h:90-96).  In this library DEFAULT selects the
 * plain CUDA path; the RVV strategies are not provided and set_algo reports
 * RVSP_ERROR_UNSUPPORTED_BACKEND for them, exactly as a non-vector build of
 * the reference does. */
typedef enum {
    RVSP_SPGEMM_ALGO_DEFAULT = 0,
    RVSP_SPGEMM_ALGO_RVV,
    RVSP_SPGEMM_ALGO_CONTIG,
    RVSP_SPGEMM_ALGO_ADAPTIVE,
    /* Plain GPU Gustavson: binned symbolic pass, device scan, numeric pass. */
    RVSP_SPGEMM_ALGO_CUDA_PLAIN = 16,
    /* Learned binning: an MLP predicts each row's output size and accumulator
     * class; symbolic and numeric fuse into one pass at the predicted
     * capacity, and overflowing rows are redone by the plain path. */
    RVSP_SPGEMM_ALGO_CUDA_LEARNED = 17
} rvsp_spgemm_algo_t;

/* The row-binning model of the learned path (new; see rvsp_cuda.h). */
typedef struct rvsp_mlp *rvsp_mlp_t;

/* Where the arrays handed to the descriptor API live (new). */
typedef enum {
    RVSP_MEM_HOST = 0,
    RVSP_MEM_DEVICE = 1
} rvsp_memory_space_t;

/* Phases timed by the optional per-descriptor profiler (new). */
typedef enum {
    RVSP_PHASE_ROWSTATS = 0,
    RVSP_PHASE_SYMBOLIC,
    RVSP_PHASE_SCAN,
    RVSP_PHASE_NUMERIC,
    RVSP_PHASE_PREDICT,
    RVSP_PHASE_FUSED,
    RVSP_PHASE_COMPACT,
    RVSP_PHASE_COPY,
    RVSP_PHASE_CHECK,
    RVSP_PHASE_COUNT
} rvsp_phase_t;

#ifdef __cplusplus
}
#endif

#endif /* RV_SPARSE_TYPES_H */
