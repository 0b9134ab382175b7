/*
 * Host allocations of the library, with a failure hook for tests.
 *
 * Every host buffer the library allocates comes from rvsp_malloc /
 * rvsp_calloc / rvsp_realloc.  rvsp_debug_fail_host_alloc(n) (rvsp_debug.h)
 * lets the next n of them succeed and makes the one after return NULL, once,
 * so a test can walk every allocation of a call and check that each failure
 * comes back as RVSP_ERROR_ALLOCATION_FAILED with nothing leaked or half
 * written.  Off (-1) by default: one relaxed atomic load per allocation.
 */
#include <stdatomic.h>
#include <stdlib.h>

#include "rvsp_debug.h"
#include "rvsp_internal.h"

static atomic_int g_fail_after = -1;
static atomic_llong g_host_allocs = 0;

/* 1 when this allocation is the one to fail. */
static int inject(void)
{
    atomic_fetch_add_explicit(&g_host_allocs, 1, memory_order_relaxed);
    int cur = atomic_load_explicit(&g_fail_after, memory_order_relaxed);
    while (cur >= 0) {
        if (atomic_compare_exchange_weak(&g_fail_after, &cur, cur - 1))
            return cur == 0;
    }
    return 0;
}

void *rvsp_malloc(size_t n)
{
    return inject() ? NULL : malloc(n);
}

void *rvsp_calloc(size_t n, size_t size)
{
    return inject() ? NULL : calloc(n, size);
}

void *rvsp_realloc(void *p, size_t n)
{
    return inject() ? NULL : realloc(p, n);
}

void rvsp_debug_fail_host_alloc(int32_t after)
{
    atomic_store(&g_fail_after, after < 0 ? -1 : (int)after);
}

int64_t rvsp_debug_host_allocs(void)
{
    return (int64_t)atomic_load(&g_host_allocs);
}
