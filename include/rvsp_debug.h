/*
 * rv-sparse-b200: test hooks (new; no reference counterpart).
 *
 * Failure injection on the host, for tests of the library's error paths: no
 * GPU fault is ever provoked.  Process-wide and thread-safe; off by default.
 */
#ifndef RVSP_DEBUG_H
#define RVSP_DEBUG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The next `after` host allocations of the library succeed and the one after
 * returns NULL (once; later ones succeed again).  after < 0 turns the hook
 * off.  The call that meets the failure returns RVSP_ERROR_ALLOCATION_FAILED
 * and frees what it had allocated. */
void rvsp_debug_fail_host_alloc(int32_t after);

/* Host allocations the library has made since the process started (failed
 * ones included), so a test can count a call's allocations and fail each. */
int64_t rvsp_debug_host_allocs(void);

#ifdef __cplusplus
}
#endif

#endif /* RVSP_DEBUG_H */
