// Per-thread K-way merge lists of the merge classes (k_merge.cu), shared
// with the persistent numeric kernel (k_persist.cu).  See k_merge.cu for the
// method: one thread merges the K sorted B rows of its row, taking the
// smallest head column each step; each list holds its next entry ahead.
#pragma once

#include <climits>

#include "device_common.cuh"
#include "kernels.cuh"

namespace rvsp {
namespace merge {

template <int K>
struct Lists {
  int32_t pos[K];  // position of the head in B
  int32_t end[K];
  int32_t cur[K];  // head column (INT_MAX when the list is done)
  int32_t nxt[K];  // column after the head (INT_MAX past the end)
  float curv[K];   // head value, next value (numeric pass)
  float nxtv[K];
  float a[K];
};

__device__ __forceinline__ void prefetch_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Opens the row's lists.  Every load here is independent of the others, and
// the lines holding each B row (both ends, columns and values) are
// prefetched into L1 so the lookahead loads hit L1.
template <int K, bool kValues>
__device__ __forceinline__ void open_lists(const Operands &op, int32_t p0,
                                           int32_t k, Lists<K> &L) {
#pragma unroll
  for (int j = 0; j < K; ++j) {
    L.cur[j] = INT_MAX;
    L.nxt[j] = INT_MAX;
    L.pos[j] = 0;
    L.end[j] = 0;
    L.a[j] = 0.0f;
    L.curv[j] = 0.0f;
    L.nxtv[j] = 0.0f;
    if (j < k) {
      const int32_t kk = __ldg(op.a_col + p0 + j);
      if (kValues) L.a[j] = __ldg(op.a_val + p0 + j);
      const int32_t b0 = __ldg(op.b_rp + kk);
      const int32_t b1 = __ldg(op.b_rp + kk + 1);
      L.pos[j] = b0;
      L.end[j] = b1;
      if (b0 < b1) {
        prefetch_l1(op.b_col + b1 - 1);
        if (kValues) prefetch_l1(op.b_val + b1 - 1);
        L.cur[j] = __ldg(op.b_col + b0);
        if (kValues) L.curv[j] = __ldg(op.b_val + b0);
        if (b0 + 1 < b1) {
          L.nxt[j] = __ldg(op.b_col + b0 + 1);
          if (kValues) L.nxtv[j] = __ldg(op.b_val + b0 + 1);
        }
      }
    }
  }
}

// Moves list j past its head: the lookahead entry becomes the head and the
// entry after it is loaded.
template <int K, bool kValues>
__device__ __forceinline__ void advance(const Operands &op, Lists<K> &L, int j) {
  const int32_t p = ++L.pos[j];
  L.cur[j] = L.nxt[j];
  if (kValues) L.curv[j] = L.nxtv[j];
  if (p + 1 < L.end[j]) {
    L.nxt[j] = __ldg(op.b_col + p + 1);
    if (kValues) L.nxtv[j] = __ldg(op.b_val + p + 1);
  } else {
    L.nxt[j] = INT_MAX;
  }
}

template <int K>
__device__ __forceinline__ int32_t min_head(const Lists<K> &L) {
  int32_t m = L.cur[0];
#pragma unroll
  for (int j = 1; j < K; ++j) m = min(m, L.cur[j]);
  return m;
}

}  // namespace merge
}  // namespace rvsp
