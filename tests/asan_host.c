/*
 * Host-layer memory check: built with -fsanitize=address against the ASan
 * build of the library (make -C rv-sparse_b200 asan) and run by
 * tests/test_asan_host.py with leak detection on.  It drives the host C
 * layer through the calls that need no GPU to reach their error paths:
 * argument errors, the Matrix Market reader, the one-shot (FP32, FP64,
 * INT8 -> INT32), descriptor and batch entry points up to their first device
 * step, and every host allocation of the reader and of the one-shot failed in
 * turn (rvsp_debug.h).  Exit 0 when every
 * status is the expected one; AddressSanitizer exits non-zero on a memory
 * error or a leak.  With a GPU present the device steps succeed instead, and
 * the driver frees what they return.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "rv_sparse.h"
#include "rvsp_debug.h"

static int failures = 0;

#define EXPECT(cond, what)                                   \
    do {                                                     \
        if (!(cond)) {                                       \
            fprintf(stderr, "asan_host: FAILED %s\n", what); \
            failures++;                                      \
        }                                                    \
    } while (0)

static const char kText[] = "%%MatrixMarket matrix coordinate real general\n"
                            "% comment\n"
                            "4 5 6\n"
                            "1 1 1.5\n2 3 -2.0\n4 5 3.25\n1 2 0.5\n3 3 1.0\n1 1 2.0\n";

static int empty(const rvsp_csr_matrix_t *m)
{
    return m->rows == 0 && m->nnz == 0 && !m->row_ptr && !m->col_idx && !m->values &&
           m->owns_data == 0;
}

/* the device step: success with a GPU, a backend or device error without */
static int device_outcome(rvsp_status_t st)
{
    return st == RVSP_SUCCESS || st == RVSP_ERROR_UNSUPPORTED_BACKEND ||
           st == RVSP_ERROR_DEVICE;
}

static void walk_parse(rvsp_memory_space_t space)
{
    rvsp_csr_matrix_t m;
    const int64_t before = rvsp_debug_host_allocs();
    rvsp_status_t st = rvsp_csr_parse_mtx(kText, sizeof(kText) - 1, space, &m);
    const int64_t n = rvsp_debug_host_allocs() - before;
    EXPECT(device_outcome(st), "parse_mtx baseline");
    if (st == RVSP_SUCCESS)
        rvsp_csr_destroy(&m);
    EXPECT(n >= 4, "parse_mtx host allocations");
    for (int64_t k = 0; k < n; k++) {
        rvsp_debug_fail_host_alloc((int32_t)k);
        st = rvsp_csr_parse_mtx(kText, sizeof(kText) - 1, space, &m);
        EXPECT(st == RVSP_ERROR_ALLOCATION_FAILED, "parse_mtx injected failure");
        EXPECT(empty(&m), "parse_mtx output empty after failure");
    }
    rvsp_debug_fail_host_alloc(-1);
}

/* Every host allocation of one one-shot product failed in turn: each must
 * return ALLOCATION_FAILED with C left empty (the reference nulls C on any
 * failure, spgemm.c:117-130). */
static void walk_oneshot(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                         const rvsp_spgemm_options_t *opts, const char *what)
{
    rvsp_csr_matrix_t C;
    memset(&C, 0, sizeof(C));
    const int64_t before = rvsp_debug_host_allocs();
    rvsp_status_t st = rvsp_spgemm_csr(A, B, &C, opts);
    const int64_t n = rvsp_debug_host_allocs() - before;
    EXPECT(device_outcome(st), what);
    if (st == RVSP_SUCCESS)
        rvsp_csr_destroy(&C);
    for (int64_t k = 0; k < n; k++) {
        memset(&C, 0, sizeof(C));
        rvsp_debug_fail_host_alloc((int32_t)k);
        st = rvsp_spgemm_csr(A, B, &C, opts);
        EXPECT(st == RVSP_ERROR_ALLOCATION_FAILED, what);
        EXPECT(empty(&C), what);
        if (st == RVSP_SUCCESS)
            rvsp_csr_destroy(&C);
    }
    rvsp_debug_fail_host_alloc(-1);
}

static void walk_read(void)
{
    char path[] = "/tmp/rvsp_asan_XXXXXX";
    int fd = mkstemp(path);
    EXPECT(fd >= 0, "mkstemp");
    if (fd < 0)
        return;
    EXPECT(write(fd, kText, sizeof(kText) - 1) == (ssize_t)(sizeof(kText) - 1), "write");
    close(fd);
    rvsp_csr_matrix_t m;
    const int64_t before = rvsp_debug_host_allocs();
    rvsp_status_t st = rvsp_csr_read_mtx(path, RVSP_MEM_HOST, &m);
    const int64_t n = rvsp_debug_host_allocs() - before;
    EXPECT(device_outcome(st), "read_mtx baseline");
    if (st == RVSP_SUCCESS)
        rvsp_csr_destroy(&m);
    for (int64_t k = 0; k < n; k++) {
        rvsp_debug_fail_host_alloc((int32_t)k);
        st = rvsp_csr_read_mtx(path, RVSP_MEM_HOST, &m);
        EXPECT(st == RVSP_ERROR_ALLOCATION_FAILED, "read_mtx injected failure");
        EXPECT(empty(&m), "read_mtx output empty after failure");
    }
    rvsp_debug_fail_host_alloc(-1);
    EXPECT(rvsp_csr_read_mtx("/nonexistent/rvsp.mtx", RVSP_MEM_HOST, &m) ==
               RVSP_ERROR_INVALID_ARGUMENT, "read_mtx missing file");
    unlink(path);
}

int main(void)
{
    /* A (2x3) and B (3x2), canonical */
    int32_t arp[] = {0, 2, 3}, aci[] = {0, 2, 1};
    float av[] = {1.0f, 2.0f, 3.0f};
    int32_t brp[] = {0, 1, 2, 4}, bci[] = {1, 0, 0, 1};
    float bv[] = {4.0f, 5.0f, 6.0f, 7.0f};
    rvsp_csr_matrix_t A, B, C;
    EXPECT(rvsp_csr_create(&A, 2, 3, 3, arp, aci, av, RVSP_DTYPE_FP32) == RVSP_SUCCESS,
           "csr_create A");
    EXPECT(rvsp_csr_create(&B, 3, 2, 4, brp, bci, bv, RVSP_DTYPE_FP32) == RVSP_SUCCESS,
           "csr_create B");
    EXPECT(rvsp_csr_validate(&A) == RVSP_SUCCESS, "validate");
    EXPECT(strlen(rvsp_status_to_string(RVSP_ERROR_INVALID_CSR)) > 0, "status string");
    size_t bytes = 0;
    EXPECT(rvsp_spgemm_buffer_size(2, &bytes) == RVSP_SUCCESS, "buffer_size");

    /* one-shot: argument errors, then the product (its device step) */
    EXPECT(rvsp_spgemm_csr(NULL, &B, &C, NULL) == RVSP_ERROR_NULL_POINTER, "oneshot NULL");
    EXPECT(rvsp_spgemm_csr(&A, &A, &C, NULL) == RVSP_ERROR_INVALID_ARGUMENT, "oneshot shape");
    memset(&C, 0, sizeof(C));
    rvsp_status_t st = rvsp_spgemm_csr(&A, &B, &C, NULL);
    EXPECT(device_outcome(st), "oneshot");
    if (st == RVSP_SUCCESS)
        rvsp_csr_destroy(&C);

    /* descriptor: create (its plan is the device step) and destroy */
    rvsp_spgemm_descr_t d = NULL;
    st = rvsp_spgemm_descr_create(&d);
    EXPECT(device_outcome(st), "descr_create");
    if (st == RVSP_SUCCESS)
        rvsp_spgemm_descr_destroy(d);
    EXPECT(rvsp_spgemm_descr_create(NULL) == RVSP_ERROR_NULL_POINTER, "descr_create NULL");

    /* batch: create, add, destroy */
    rvsp_spgemm_batch_t b = NULL;
    st = rvsp_spgemm_batch_create(&b);
    EXPECT(device_outcome(st), "batch_create");
    if (st == RVSP_SUCCESS) {
        for (int i = 0; i < 40; i++)  /* past the first capacity */
            EXPECT(rvsp_spgemm_batch_add(b, &A, &B, NULL) == RVSP_SUCCESS, "batch_add");
        rvsp_spgemm_batch_destroy(b);
    }

    /* the one-shot in its three value types, every host allocation failed */
    walk_oneshot(&A, &B, NULL, "oneshot fp32 walk");
    double av64[] = {1.0, 2.0, 3.0}, bv64[] = {4.0, 5.0, 6.0, 7.0};
    int8_t av8[] = {1, 2, 3}, bv8[] = {4, 5, 6, 7};
    rvsp_csr_matrix_t A64, B64, A8, B8;
    EXPECT(rvsp_csr_create(&A64, 2, 3, 3, arp, aci, av64, RVSP_DTYPE_FP64) == RVSP_SUCCESS,
           "csr_create A64");
    EXPECT(rvsp_csr_create(&B64, 3, 2, 4, brp, bci, bv64, RVSP_DTYPE_FP64) == RVSP_SUCCESS,
           "csr_create B64");
    EXPECT(rvsp_csr_create(&A8, 2, 3, 3, arp, aci, av8, RVSP_DTYPE_INT8) == RVSP_SUCCESS,
           "csr_create A8");
    EXPECT(rvsp_csr_create(&B8, 3, 2, 4, brp, bci, bv8, RVSP_DTYPE_INT8) == RVSP_SUCCESS,
           "csr_create B8");
    const rvsp_spgemm_options_t o64 = {RVSP_BACKEND_CUDA, RVSP_DTYPE_FP64, RVSP_DTYPE_FP64};
    const rvsp_spgemm_options_t o8 = {RVSP_BACKEND_CUDA, RVSP_DTYPE_INT8, RVSP_DTYPE_INT32};
    walk_oneshot(&A64, &B64, &o64, "oneshot fp64 walk");
    walk_oneshot(&A8, &B8, &o8, "oneshot int8 walk");

    walk_parse(RVSP_MEM_HOST);
    walk_parse(RVSP_MEM_DEVICE);
    walk_read();

    if (failures)
        fprintf(stderr, "asan_host: %d check(s) failed\n", failures);
    else
        printf("asan_host: all checks passed\n");
    return failures ? 1 : 0;
}
